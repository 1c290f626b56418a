/*
 * CPU oracle harness around the reference's own hot-path sources.
 * TEST INFRASTRUCTURE ONLY: only tests/, the smoke check and the bench's CPU
 * baseline leg load the library built from this file.
 *
 * The library oracle/_ref/libhosref_M<M>.so is the reference's
 *   Csource/2dpar/hosm_2d_par.c, operators_par.c, time_schemes_par.c,
 *   fft_routines_2d_par.c
 * compiled unchanged (oracle/Makefile), with NLevs = M-1 substituted into a
 * generated copy of euler_2d_par.h:24, linked with the single-rank FFTW-MPI
 * shim (shim/shim_fft.c) and with this harness.  The harness plays the role
 * of the reference driver main_2d_par.c: it sets the globals that
 * get_params (hdf5_routines_2d_par.c:13-101) and main (main_2d_par.c:126-191)
 * would set, and exposes flat-pointer entry points so that tests can call
 * the reference's functions from Python.
 *
 * Array conventions (all double precision, host memory):
 *   physical fields: unpadded row-major [Nx][Ny] (the harness inserts the
 *     FFTW-MPI padding [Nx][Ny+2] used at fft_routines_2d_par.c:19,86);
 *   spectral fields: interleaved complex [Ny/2+1][Nx] (TRANSPOSED_OUT),
 *     alloc_local = Nx*(Ny/2+1) complex values per field;
 *   packed state u = [eta_hat | phi_hat], 2*alloc_local complex values
 *     (main_2d_par.c:150,158).
 */
#include "euler_2d_par.h"
#include "fft_routines_2d_par.h"
#include "hosm_2d_par.h"
#include "operators_par.h"
#include "time_schemes_par.h"

static int harness_ready = 0;

int ref_nlevs(void) { return NLevs; }

long ref_alloc_local(void) { return (long)alloc_local; }

/* Sets the globals the reference driver sets, creates the FFT plans and
 * calls Setup_TimeScheme / rhs_hos_setup (main_2d_par.c:126-191,252-254). */
int ref_setup(int nx, int ny, double lx, double ly, double gg, int ramp, double tramp, int scheme) {
  if (nx < 4 || ny < 4 || (nx & (nx - 1)) || (ny & (ny - 1))) return -1;
  if (harness_ready) {
    fftw_destroy_plan(fftp);
    fftw_destroy_plan(ifftp);
    fftw_free(f);
    fftw_free(hf);
  }
  mpi_rank = 0;
  mpi_size = 1;
  comm = MPI_COMM_WORLD;
  info = MPI_INFO_NULL;
  Nx = nx;
  Ny = ny;
  fNx = nx;
  fNy = ny;
  Lx = lx;
  Ly = ly;
  g = gg;
  rampflg = ramp;
  Tramp = tramp;
  /* same expressions as hdf5_routines_2d_par.c:98-99 */
  Kx0 = 2 * M_PI / Lx;
  Ky0 = 2 * M_PI / Ly;
  alloc_local = fftw_mpi_local_size_2d_transposed(fNx, fNy / 2 + 1, MPI_COMM_WORLD, &local_Nx, &local_0_start,
                                                  &local_Nyhpo, &local_1_start);
  local_N = Nx * local_Nyhpo;
  f = fftw_alloc_real(2 * alloc_local);
  hf = fftw_alloc_complex(alloc_local);
  fftp = fftw_mpi_plan_dft_r2c_2d(fNx, fNy, f, hf, MPI_COMM_WORLD, FFTW_MEASURE | FFTW_MPI_TRANSPOSED_OUT);
  ifftp = fftw_mpi_plan_dft_c2r_2d(fNx, fNy, hf, f, MPI_COMM_WORLD, FFTW_MEASURE | FFTW_MPI_TRANSPOSED_IN);
  if (!fftp || !ifftp) return -2;
  memset(runtime_data_buff, 0, sizeof(runtime_data_buff));
  strncpy(runtime_data_buff, "/dev/null", sizeof(runtime_data_buff) - 1);
  /* The reference allocates afresh on every call and never frees
   * (rhs_hos_clean is never called, hosm_2d_par.c:104-134); a test process
   * calls this a handful of times, so the leak is bounded. */
  Setup_TimeScheme(scheme);
  rhs_hos_setup();
  harness_ready = 1;
  return 0;
}

static double* pad_real(const double* u) {
  double* p = fftw_alloc_real(2 * alloc_local);
  for (ptrdiff_t x = 0; x < Nx; x++)
    for (ptrdiff_t y = 0; y < Ny; y++) p[(Ny + 2) * x + y] = u[(ptrdiff_t)Ny * x + y];
  return p;
}

static void unpad_real(const double* p, double* u) {
  for (ptrdiff_t x = 0; x < Nx; x++)
    for (ptrdiff_t y = 0; y < Ny; y++) u[(ptrdiff_t)Ny * x + y] = p[(Ny + 2) * x + y];
}

static fftw_complex* copy_spec(const double* hu, ptrdiff_t nfields) {
  fftw_complex* c = fftw_alloc_complex(nfields * alloc_local);
  memcpy(c, hu, sizeof(fftw_complex) * (size_t)(nfields * alloc_local));
  return c;
}

/* fft_2d (fft_routines_2d_par.c:21-58): normalised r2c. */
void ref_fft_2d(const double* u, double* hu) {
  double* p = pad_real(u);
  fft_2d(p, (fftw_complex*)hu, fftp);
  fftw_free(p);
}

/* ifft_2d (fft_routines_2d_par.c:68-103): unnormalised c2r. */
void ref_ifft_2d(const double* hu, double* u) {
  fftw_complex* c = copy_spec(hu, 1);
  double* p = fftw_alloc_real(2 * alloc_local);
  ifft_2d(c, p, ifftp);
  unpad_real(p, u);
  fftw_free(p);
  fftw_free(c);
}

/* Initial transform and dealiasing (main_2d_par.c:258-262). */
void ref_init_state(const double* eta, const double* phi, double* u) {
  fftw_complex* uc = (fftw_complex*)u;
  double* pe = pad_real(eta);
  double* pp = pad_real(phi);
  fft_2d(pe, uc, fftp);
  fft_2d(pp, &uc[alloc_local], fftp);
  Dealias(uc);
  Dealias(&uc[alloc_local]);
  fftw_free(pe);
  fftw_free(pp);
}

/* rhs_hos (hosm_2d_par.c:138-235). */
void ref_rhs(const double* u, double* rhs, double t) {
  fftw_complex* uc = copy_spec(u, 2);
  rhs_hos((fftw_complex*)rhs, uc, t);
  fftw_free(uc);
}

/* Zvel (hosm_2d_par.c:240-445). */
void ref_zvel(const double* u, double* wM, double* wM2, double* w2M, double* w2M2, double t) {
  fftw_complex* uc = copy_spec(u, 2);
  Zvel(uc, (fftw_complex*)wM, (fftw_complex*)wM2, (fftw_complex*)w2M, (fftw_complex*)w2M2, t);
  fftw_free(uc);
}

/* nsteps calls of sol_update_RK (time_schemes_par.c:28-121); ham[k] receives
 * the Hamiltonian the reference computes at stage 0 of step k
 * (time_schemes_par.c:73-74). */
void ref_steps(double* u, double* t, double dt, int nsteps, double* ham) {
  char dtflag[20] = {0};
  for (int k = 0; k < nsteps; k++) {
    sol_update_RK((fftw_complex*)u, t, dt, dtflag);
    if (ham) ham[k] = Ham;
  }
}

void ref_dx(const double* in, double* out) {
  fftw_complex* c = copy_spec(in, 1);
  Dx(c, (fftw_complex*)out);
  fftw_free(c);
}

void ref_dy(const double* in, double* out) {
  fftw_complex* c = copy_spec(in, 1);
  Dy(c, (fftw_complex*)out);
  fftw_free(c);
}

void ref_dz(const double* in, double* out) { Dz((const fftw_complex*)in, (fftw_complex*)out); }

void ref_mult(const double* a, const double* b, double* out) {
  fftw_complex* ca = copy_spec(a, 1);
  fftw_complex* cb = copy_spec(b, 1);
  Mult(ca, cb, (fftw_complex*)out);
  fftw_free(ca);
  fftw_free(cb);
}

void ref_sum(const double* a, const double* b, double* out) {
  fftw_complex* ca = copy_spec(a, 1);
  fftw_complex* cb = copy_spec(b, 1);
  Sum(ca, cb, (fftw_complex*)out);
  fftw_free(ca);
  fftw_free(cb);
}

void ref_dealias(double* u) { Dealias((fftw_complex*)u); }

double ref_hamiltonian(const double* eta, const double* eta_t, const double* phi) {
  return Hamiltonian((const fftw_complex*)eta, (const fftw_complex*)eta_t, (const fftw_complex*)phi);
}

double ref_rampfun(double t) { return RampFun(t); }
