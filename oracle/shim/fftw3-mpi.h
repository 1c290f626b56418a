/*
 * Single-rank FFTW-MPI shim.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference (Csource/2dpar) calls FFTW 3.3.x through FFTW-MPI with
 * FFTW_MPI_TRANSPOSED_OUT / _IN plans (main_2d_par.c:188-191) and
 * fftw_execute (fft_routines_2d_par.c:37,88).  FFTW is not installed here, so
 * the oracle links this shim instead.  It implements FFTW's documented
 * transform definitions for the 2-D real-data case on one rank:
 *
 *   r2c (unnormalised, TRANSPOSED_OUT):
 *     out[ky*Nx + kx] = sum_{ix,iy} in[ix*(Ny+2) + iy] * exp(-2 pi i (kx ix/Nx + ky iy/Ny))
 *     for ky = 0..Ny/2, kx = 0..Nx-1; the real input uses FFTW-MPI's padded
 *     row stride 2*(Ny/2+1).
 *   c2r (unnormalised, TRANSPOSED_IN):
 *     a complex inverse DFT along x for every ky column, then a 1-D
 *     complex-to-real inverse along y that ignores the imaginary parts of the
 *     ky = 0 and ky = Ny/2 bins (FFTW's halfcomplex convention).
 *
 * The transform arithmetic itself is this project's own code (shim_fft.c).
 * The pinned third-party version the reference targets is FFTW 3.3.3
 * (Makefile:18-19); only its public definitions are restated.
 */
#ifndef HOS_ORACLE_SHIM_FFTW3_MPI_H
#define HOS_ORACLE_SHIM_FFTW3_MPI_H

#include <stddef.h>
#include <complex.h>
#include "mpi.h"

typedef double _Complex fftw_complex;
typedef float _Complex fftwf_complex;

typedef struct hos_shim_plan* fftw_plan;
typedef struct hos_shim_planf* fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_IN (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)

void fftw_mpi_init(void);
ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm,
                                 ptrdiff_t* local_n0, ptrdiff_t* local_0_start);
ptrdiff_t fftw_mpi_local_size_2d_transposed(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm,
                                            ptrdiff_t* local_n0, ptrdiff_t* local_0_start,
                                            ptrdiff_t* local_n1, ptrdiff_t* local_1_start);
double* fftw_alloc_real(size_t n);
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double* in, fftw_complex* out,
                                   MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, double* out,
                                   MPI_Comm comm, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* Single-precision names appear only in the reference's non-USE_DOUBLES
 * branches; they are declared so those declarations type-check. */
float* fftwf_alloc_real(size_t n);
fftwf_complex* fftwf_alloc_complex(size_t n);
void fftwf_free(void* p);
void fftwf_execute(const fftwf_plan p);

#endif
