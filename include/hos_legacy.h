/*
 * hos_legacy.h -- the reference's hot-path entry points, exported by
 * libhos_gpu.so with their original names and signatures, so that the
 * reference's host driver (Csource/2dpar/main_2d_par.c) links against the
 * library in place of time_schemes_par.o, hosm_2d_par.o, operators_par.o and
 * fft_routines_2d_par.o.
 *
 * The reference declares these with fftw_complex* (double _Complex*) and
 * TYPE_REAL = double (built with USE_DOUBLES, Makefile.Nicole:10-16); here
 * the complex arrays are declared as double* to interleaved (re, im) pairs,
 * which is the same ABI.  The reference's callers include their own headers
 * and never this one.
 *
 * Like the reference, these functions take their sizes and constants from
 * process-global variables (euler_2d_par.h:40-98, fft_routines_2d_par.h:
 * 17-38), which the driver sets: Nx, Ny, Lx, Ly, Kx0, Ky0, g, rampflg,
 * Tramp, alloc_local, local_N, local_Nyhpo, local_1_start, mpi_rank,
 * runtime_data_buff.  The library defines them too (so that it loads on its
 * own); a driver's definitions take precedence at link time.  Only a single
 * rank (local_1_start = 0, local_Nyhpo = Ny/2+1) is supported: every field
 * lives on one GPU.
 *
 * The HOS order is a compile-time constant in the reference (NLevs,
 * euler_2d_par.h:24).  Here it is NLevs = 2 by default and set with
 * hos_legacy_set_nlevs() or the environment variable HOS_NLEVS.
 *
 * Arrays are host memory.  sol_update_RK uploads the state, advances one
 * step on the GPU and downloads it (the state is correct on the host after
 * every call), unless resident mode (below) keeps it on the GPU.  Errors are recorded for hos_last_error(); the functions
 * return void, as the reference's do.
 */
#ifndef HOS_LEGACY_H
#define HOS_LEGACY_H

#ifdef __cplusplus
extern "C" {
#endif

/* Setup_TimeScheme, time_schemes_par.c:127-314 (ids 1..5: RK45-DP, RK4, Euler, midpoint, Heun). */
void Setup_TimeScheme(int scheme_flg);

/* sol_update_RK, time_schemes_par.c:28-121: one RK step of the packed state u
 * (2*alloc_local complex), *t += dt; appends "t Ham" to runtime_data_buff as
 * time_schemes_par.c:73-93 does. */
void sol_update_RK(double* u, double* t, double dt, char* dtflag);

/* rhs_hos_setup / rhs_hos_clean, hosm_2d_par.c:51-134: create / release the
 * GPU context for the current globals. */
void rhs_hos_setup(void);
void rhs_hos_clean(void);

/* rhs_hos, hosm_2d_par.c:138-235. */
void rhs_hos(double* hrhs, double* hu, double t);

/* rhs_test, hosm_2d_par.c:36-45: linear advection (Dx of eta, Dy of phi). */
void rhs_test(double* hrhs, double* hu);

/* Zvel, hosm_2d_par.c:240-445. */
void Zvel(double* hu, double* hZvelM, double* hZvelM2, double* hZvel2M, double* hZvel2M2, double t);

/* ZvelLinear, hosm_2d_par.c:448-455: Dz of the phi field. */
void ZvelLinear(const double* hu, double* hZvelLinear);

/* Hamiltonian, hosm_2d_par.c:462-523. */
double Hamiltonian(const double* heta, const double* heta_t, const double* hphi);

/* RampFun, hosm_2d_par.c:526-530. */
double RampFun(const double t);

/* Spectral operators, operators_par.c:20-325. */
void Dx(double* hu, double* hu_x);
void Dy(double* hu, double* hu_y);
void Dz(const double* hu, double* hu_z);
void Mult(double* hu1, double* hu2, double* hprod);
void Sum(double* hu1, double* hu2, double* hsum);
void Dealias(double* hu);

/* fft_2d / ifft_2d, fft_routines_2d_par.c:21-103.  u is the padded real
 * array [Nx][Ny+2] the reference uses; the plan argument is ignored. */
void fft_2d(double* u, double* hu, void* plan);
void ifft_2d(double* hu, double* u, void* plan);

/* Sets the HOS order of the legacy context (NLevs = M - 1, default 2). */
void hos_legacy_set_nlevs(int nlevs);

/* Resident mode (off by default; on with hos_legacy_set_resident(1) or
 * HOS_LEGACY_RESIDENT=1 in the environment): the state array passed to
 * sol_update_RK stays on the GPU between calls instead of being uploaded and
 * downloaded every step.  The host array is brought up to date when one of
 * the functions here reads it (ifft_2d at a save, Hamiltonian, Zvel, ...),
 * at rhs_hos_clean() and by hos_legacy_sync(); a function here that writes
 * into it (Dealias, fft_2d, ...) makes the host copy the one the next step
 * uploads.  The reference's driver reads the state only through ifft_2d
 * (main_2d_par.c:310-311), so it can run in this mode unchanged; code that
 * reads the array directly calls hos_legacy_sync() first. */
void hos_legacy_set_resident(int on);
void hos_legacy_sync(void);

#ifdef __cplusplus
}
#endif

#endif /* HOS_LEGACY_H */
