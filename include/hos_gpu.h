/*
 * hos_gpu.h -- C ABI of the B200 (sm_100a) HOS time-advance library
 * (libhos_gpu.so).
 *
 * Two groups of entry points live in the library.
 *
 * 1. Handle API (this header).  A handle owns one wave field (or one ensemble
 *    member): its FP64 spectral state resident in GPU memory, its scratch,
 *    its CUDA stream and its captured step graph.  Every call returns an int
 *    status (HOS_OK or an HOS_ERR_* code); hos_last_error() describes the
 *    most recent failure of the calling thread.  Calls on one handle must not
 *    overlap; different handles may be driven from different threads.
 *
 * 2. Reference-compatible symbols (hos_legacy.h): the functions of the
 *    reference's Csource/2dpar hot path with their original signatures, so
 *    that the unchanged host driver main_2d_par.c links against this library
 *    in place of time_schemes_par.o, hosm_2d_par.o, operators_par.o and
 *    fft_routines_2d_par.o.
 *
 * Array conventions (host or device, always double precision at the ABI):
 *   physical field : real [nx][ny], row-major (x major, y contiguous), unpadded;
 *   spectral field : complex [ny/2+1][nx] as interleaved (re, im) doubles --
 *                    the reference's single-rank FFTW_MPI_TRANSPOSED_OUT
 *                    layout (main_2d_par.c:189, Dx at operators_par.c:66);
 *   packed state   : [eta_hat | phi_hat], two spectral fields back to back
 *                    (main_2d_par.c:150,158; sol_update_RK's u).
 * Spectral fields are normalised by 1/(nx*ny) as fft_2d does
 * (fft_routines_2d_par.c:53-55).
 */
#ifndef HOS_GPU_H
#define HOS_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  HOS_OK = 0,
  HOS_ERR_ARG = 1,       /* invalid argument (size, order, scheme, null pointer) */
  HOS_ERR_CUDA = 2,      /* a CUDA call failed */
  HOS_ERR_NOMEM = 3,     /* device memory exhausted */
  HOS_ERR_NONFINITE = 4, /* the state contains NaN or Inf */
  HOS_ERR_STATE = 5,     /* call not valid in the handle's current state */
  HOS_ERR_TIMEOUT = 6,   /* a bounded wait ran out */
  HOS_ERR_BUSY = 7       /* admission refused (no slot or memory) */
};

enum { HOS_PREC_FP64 = 0, HOS_PREC_FP32 = 1 };

/* Runge-Kutta scheme ids of Setup_TimeScheme (time_schemes_par.c:127-314). */
enum { HOS_RK45DP = 1, HOS_RK4 = 2, HOS_EULER = 3, HOS_MIDPOINT = 4, HOS_HEUN = 5 };

typedef struct hos_params {
  int nx, ny;       /* grid, powers of two, 16 <= nx <= 4096, 16 <= ny <= 4096 */
  double lx, ly;    /* domain lengths (Kx0 = 2 pi / Lx, hdf5_routines_2d_par.c:98-99) */
  double g;         /* gravity */
  int order;        /* HOS order M = NLevs + 1 (euler_2d_par.h:24), 1..7 */
  int precision;    /* HOS_PREC_FP64 (drop-in) or HOS_PREC_FP32 (FP32 transforms, FP64 state) */
  double depth;     /* <= 0: deep water (the reference); > 0: finite depth h */
  int rampflg;      /* Dommermuth ramp on/off (hosm_2d_par.c:211-229) */
  double tramp;     /* ramp time scale Tramp */
  int scheme;       /* HOS_RK4 etc. */
  int mx, my;       /* dealias bounds; 0 selects the reference rule (operators_par.c:290-291) */
  int tune[8];      /* kernel shapes (0 = default): elements per thread of the x-inverse, x-forward,
                       (level) y-inverse and y-forward passes (8, 16, or 32 in FP32), then the base-2 exponents
                       scaling their lines per block; chosen by hos_b200.autotune */
  int tune_opb;     /* z-derivative orders per block of the level x-forward pass (0 = all in one block) */
  int tune_nofuse;  /* 1: run each level's y-forward pass as its own launch instead of inside the
                       previous level's y-inverse pass */
  int tune_ys;      /* elements per thread of the stage y-inverse pass (0: as the level y-inverse, tune[2]) */
  int tune_sys;     /* its lines-per-block exponent (used when tune_ys is set) */
} hos_params;

typedef struct hos_ctx* hos_handle;

/* Fills p with the reference defaults for an nx x ny grid (M = 3, RK4,
 * FP64, deep water, no ramp, 2 pi x 2 pi, g = 1). */
void hos_default_params(hos_params* p, int nx, int ny);

/* Creates a handle on the current CUDA device and a stream of its own.
 * Replaces the allocations of rhs_hos_setup (hosm_2d_par.c:51-97) and
 * Setup_TimeScheme (time_schemes_par.c:127-196). */
int hos_create(const hos_params* p, hos_handle* out);
int hos_destroy(hos_handle h);

/* Device bytes a handle with these parameters allocates (admission control). */
size_t hos_footprint_bytes(const hos_params* p);

/* Device memory a new handle can take on the current device: the driver's
 * free memory plus what the stream-ordered pool that handles allocate from
 * holds unused (memory of destroyed handles, kept up to HOS_POOL_KEEP_MB,
 * 8 GiB by default, for the next handles). */
int hos_device_free_bytes(size_t* free_bytes);

/* Dealias bounds in effect (mx, my) for a handle. */
int hos_get_bounds(hos_handle h, int* mx, int* my);

/* State transfer.  *_spectral take/return the packed state (2*(ny/2+1)*nx
 * complex).  set_state_physical applies fft_2d and Dealias to eta and phi
 * exactly as main_2d_par.c:258-262; get_state_physical applies ifft_2d as
 * main_2d_par.c:310-311.  Pointers may be host (pageable or pinned) or
 * device memory. */
int hos_set_state_spectral(hos_handle h, const double* u, double t);
int hos_get_state_spectral(hos_handle h, double* u, double* t);
int hos_set_state_physical(hos_handle h, const double* eta, const double* phi, double t);
int hos_get_state_physical(hos_handle h, double* eta, double* phi);

/* Advances nsteps RK steps of size dt on the device (sol_update_RK,
 * time_schemes_par.c:28-121, called nsteps times).  Asynchronous with
 * respect to the host; hos_sync waits. */
int hos_step(hos_handle h, double dt, int nsteps);
/* Adaptive steps with the reference's Dormand-Prince pair (scheme 1,
 * Setup_TimeScheme, time_schemes_par.c:183-235), from the handle's time to
 * t_end.  Each step advances with the 4th-order weights c, as the
 * reference's fixed-step scheme 1 does; the 5th-order weights cs, which the
 * reference computes but never uses, give the error estimate
 * e = dt sum_s (c_s - cs_s) k_s.  A step is kept when
 * max|e| <= atol + rtol max|u| (complex moduli over the packed state u after
 * the step); otherwise the state, time and step count return to the step's
 * start.  The next step is dt * min(5, max(0.2, 0.9 (max|e| / tol)^(-1/5))),
 * and the last is shortened to land on t_end.  *dt is the first trial step
 * on entry and the next proposed step on return.  Synchronous; the energy
 * record holds the kept steps.  HOS_ERR_STATE if the scheme is not 1 or
 * max_steps attempts did not reach t_end. */
int hos_step_adaptive(hos_handle h, double t_end, double* dt, double rtol, double atol, int max_steps,
                      int* accepted, int* rejected);
/* Waits for the handle's work.  Returns HOS_ERR_NONFINITE when a step's
 * energy was NaN or Inf, i.e. the state became non-finite (set on the device
 * by the step-end reduction; cleared by the next hos_set_state_*). */
int hos_sync(hos_handle h);
/* First step whose energy was not finite, or -1 (steps are counted from
 * hos_create: 0 is the handle's first step). */
int hos_health(hos_handle h, long long* first_nonfinite_step);
/* Test hook: the device allocations after the next `after` ones fail with
 * HOS_ERR_NOMEM (the call that hits it frees what it had allocated);
 * after < 0 turns it off.  HOS_FAIL_ALLOC_AFTER in the environment sets the
 * initial value. */
void hos_inject_alloc_failure(long after);

/* Stage-0 Hamiltonian of each step (hosm_2d_par.c:462-523, logged by the
 * reference to runtime.dat at time_schemes_par.c:73-93) and the step-start
 * time it belongs to, oldest first.  Returns the number of records written
 * in *count (at most max).  hos_clear_history empties the record. */
int hos_energy_history(hos_handle h, double* t_out, double* ham_out, int max, int* count);
int hos_clear_history(hos_handle h);

/* One right-hand-side evaluation rhs_hos(rhs, u, t) (hosm_2d_par.c:138-235)
 * on a packed spectral state; does not touch the handle's state. */
int hos_rhs(hos_handle h, const double* u, double* rhs, double t);

/* fft_2d / ifft_2d (fft_routines_2d_par.c:21-103) on the handle's grid:
 * normalised r2c of a physical field and unnormalised c2r of a spectral one. */
int hos_fft_2d(hos_handle h, const double* u_phys, double* hu);
int hos_ifft_2d(hos_handle h, const double* hu, double* u_phys);
/* The same with a physical row stride of ld >= ny doubles (the reference's
 * padded layout has ld = ny + 2, fft_routines_2d_par.c:19,86). */
int hos_fft_2d_ld(hos_handle h, const double* u_phys, int ld, double* hu);
int hos_ifft_2d_ld(hos_handle h, const double* hu, double* u_phys, int ld);

/* Zvel (hosm_2d_par.c:240-445) on a packed spectral state: the spectral
 * W^(M), W^(M-2), (W^2)^(M), (W^2)^(M-2), each one field [ny/2+1][nx]. */
int hos_zvel(hos_handle h, const double* u, double* wM, double* wM2, double* w2M, double* w2M2);

/* The spectral operators of operators_par.c on one field [ny/2+1][nx]:
 * Dx (:20-75), Dy (:85-120), Dz (:130-196; |k| tanh(|k|h) for finite
 * depth), Dealias (:283-325), Sum (:247-279, uses b) and Mult (:210-235,
 * uses b: c2r both, multiply, normalised r2c). */
enum { HOS_OP_DX = 0, HOS_OP_DY = 1, HOS_OP_DZ = 2, HOS_OP_DEALIAS = 3, HOS_OP_SUM = 4, HOS_OP_MULT = 5 };
int hos_spectral_op(hos_handle h, int op, const double* a, const double* b, double* out);

/* Hamiltonian (hosm_2d_par.c:462-523) of spectral eta, eta_t, phi. */
int hos_hamiltonian(hos_handle h, const double* eta, const double* eta_t, const double* phi, double* H);

/* Whether the resident state is finite (1) or holds NaN/Inf (0). */
int hos_check_finite(hos_handle h, int* finite);

/* Volume (the k = 0 mode of eta_hat, real part) of the resident state. */
int hos_volume(hos_handle h, double* vol);

/* Per-pass timing of one RK stage on the resident state (written to
 * scratch; the state is untouched).  Each pass kind gets one record: the
 * number of its launches in a stage, the mean duration of a launch (CUDA
 * events on the handle's stream, averaged over reps) and the algorithmic
 * bytes of a launch (what the pass must read plus write). */
typedef struct hos_pass_stat {
  char name[32];
  int launches_per_stage;
  double ms_per_launch;
  double bytes_per_launch;
} hos_pass_stat;
int hos_profile_stage(hos_handle h, double dt, int reps, hos_pass_stat* out, int max, int* count);

/* Ensembles (many independent fields advanced together).  Members are
 * existing handles of any grid, order, precision and dt; members with the
 * same grid, precision and scheme form a size class whose every pass is one
 * launch over all its members (blockIdx.z = member), and one RK step of all
 * classes is one CUDA graph with the classes on parallel streams.  Each
 * member advances exactly as hos_step(member, dt[i], 1) would, and keeps
 * its own state, time and energy record.  No counterpart in the reference
 * (it advances one field per process). Members must not be stepped on their
 * own while the ensemble exists; call hos_ensemble_sync before reading them. */
typedef struct hos_ens* hos_ensemble;
/* Classes mode (as above). */
int hos_ensemble_create(const hos_handle* members, const double* dt, int n, hos_ensemble* out);
/* mode HOS_ENS_CLASSES: as hos_ensemble_create.  mode HOS_ENS_PERSISTENT:
 * one RK step of all members is ONE launch of a persistent kernel whose
 * resident blocks take work items (blocks of one pass of one member) from a
 * device list and wait, with a bounded wait, for the member's earlier
 * passes; members of every grid, order, precision and depth share it.  Its
 * members must have grids of 64..2048 points per direction and the default
 * kernel shapes; each member ends bitwise as hos_step would leave it.  A
 * wait that runs out makes hos_ensemble_sync return HOS_ERR_TIMEOUT (the
 * members' states are then not valid until set again).  No counterpart in
 * the reference (time_schemes_par.c:28-121 advances one field per process). */
enum { HOS_ENS_CLASSES = 0, HOS_ENS_PERSISTENT = 1 };
int hos_ensemble_create_ex(const hos_handle* members, const double* dt, int n, int mode, hos_ensemble* out);
/* Per-member step budgets (either mode).  steps[i] >= 0 lets member
 * i take that many more steps, after which its work items are skipped (its
 * state and time stay as they are) until a new budget is set; -1 (the value
 * after create) sets no limit.  get_remaining reads what is left (after the
 * queued steps; it synchronises the ensemble's stream). */
int hos_ensemble_set_steps(hos_ensemble e, const int* steps);
int hos_ensemble_get_remaining(hos_ensemble e, int* steps);
/* Bound of one wait of the persistent kernel, nanoseconds (default 2 s). */
int hos_ensemble_set_wait_limit(hos_ensemble e, long long ns);
/* Failure injection for tests: on != 0 re-plans the work list so that one
 * task of the first member waits for one more completed item than its
 * earlier passes have, so the wait runs out and the step fails with
 * HOS_ERR_TIMEOUT; on = 0 restores the plan. */
int hos_ensemble_withhold_dependency(hos_ensemble e, int on);
int hos_ensemble_step(hos_ensemble e, int nsteps);
int hos_ensemble_sync(hos_ensemble e);
int hos_ensemble_info(hos_ensemble e, int* nclasses, int* launches_per_step);
/* The stream the ensemble's step graphs are launched on (cudaStream_t). */
void* hos_ensemble_stream(hos_ensemble e);
int hos_ensemble_destroy(hos_ensemble e);

/* Kernel launches of this library in one RK step of the handle. */
int hos_launches_per_step(hos_handle h);

/* The normalised 2-D real-to-complex transform of fft_2d for callers that
 * cannot allocate GPU memory: code running while a stream is captured into a
 * CUDA graph (cudaMalloc/cudaFree are not permitted there), latency-critical
 * loops in which an allocation would synchronise the device, and hosts whose
 * own allocator owns all device memory.  No counterpart in the reference:
 * it is this library's addition.  u_phys (real [nx][ny]) and hu (complex
 * [ny/2+1][nx], interleaved) are device pointers; the transform runs on
 * `stream` (a cudaStream_t, 0 for the default stream) and nothing is
 * allocated or freed: the intermediate lives in a fixed device array of the
 * library (about 8.5 MB per GPU, held until exit).  Limits: nx, ny powers of
 * two in [16, 2048] and nx*(ny/2+1) <= 525312 (e.g. 1024 x 1024); larger
 * grids return HOS_ERR_ARG.  The first call on a device looks up that
 * array's device address and should come before any stream capture.  All
 * calls on a device share the array, so calls that overlap on the GPU race;
 * order them on one stream. */
int hos_fft_2d_noalloc(const double* u_phys, double* hu, int nx, int ny, void* stream);

/* ------------------------------------------------------------------ HDF5 files
 * The subset of the HDF5 format the driver's files use, without libhdf5:
 * superblock v0/v1, root-group datasets with version 1 object headers,
 * contiguous or compact storage.  Replaces get_params / get_ic_2d
 * (hdf5_routines_2d_par.c:13-101, :104-188), which read every dataset as
 * H5T_IEEE_F64LE whatever its stored type (integers and floats convert), and
 * the snapshot writers (write_header_2d :227-283, write_field_2d :286-392,
 * write_coordinates_2d :395-446, write_extra_2d :449-537), which write 1x1
 * header datasets and [Nx][Ny] fields into a new file.  Errors (missing file
 * or dataset, unsupported storage, size mismatch) return HOS_ERR_ARG with
 * the reason in hos_last_error(). */
enum { HOS_H5_F64 = 0, HOS_H5_F32 = 1, HOS_H5_I64 = 2, HOS_H5_I32 = 3 };
/* Names of the root group's datasets, one per line, into names[cap]. */
int hos_h5_list(const char* path, char* names, int cap, int* count);
/* Rank, dimensions (up to 4) and stored type (HOS_H5_*, -1 for other sizes). */
int hos_h5_info(const char* path, const char* name, int* rank, long long* dims, int* type);
/* Reads all nelems elements (row-major) as doubles. */
int hos_h5_read_f64(const char* path, const char* name, double* out, long long nelems);
/* Writes a new file (replacing any) holding n datasets of rank 0..2:
 * dims[2*i..2*i+1] are dataset i's dimensions, data[i] its little-endian
 * elements of type types[i] (HOS_H5_F64, HOS_H5_F32 or HOS_H5_I64). */
int hos_h5_write(const char* path, int n, const char* const* names, const void* const* data, const int* types,
                 const int* ranks, const long long* dims);

/* CUDA stream of the handle (a cudaStream_t), for callers that order their
 * own work against it. */
void* hos_stream(hos_handle h);

/* Message of the last failed call on this thread ("" if none). */
const char* hos_last_error(void);

/* Library build description (kernel set, architecture). */
const char* hos_version(void);

#ifdef __cplusplus
}
#endif

#endif /* HOS_GPU_H */
