/*
 * fftw3-mpi.h -- the FFTW-MPI calls of the reference's host driver, for a
 * driver linked against libhos_gpu.so on a host without FFTW.
 *
 * With the library in place of fft_routines_2d_par.o, the driver uses FFTW
 * only to size and allocate its arrays and to create the two plans it hands
 * to fft_2d / ifft_2d (main_2d_par.c:132-191), which the library ignores.
 * libhos_hostshim.so implements these for one rank: the local sizes are the
 * whole grid (TRANSPOSED layout [Ny/2+1][Nx]), allocations are 64-byte
 * aligned and may be released with free() (main_2d_par.c:366), and a plan
 * records its sizes.  Executing a plan on the host is not offered: the
 * transforms run on the GPU through fft_2d / ifft_2d, and fftw_execute
 * reports that and ends the program.  A host that has FFTW-MPI uses its own
 * header and library instead.
 */
#ifndef HOS_HOSTSHIM_FFTW3_MPI_H
#define HOS_HOSTSHIM_FFTW3_MPI_H

#include <stddef.h>
#ifndef __cplusplus
#include <complex.h>
#endif
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
#else
typedef double _Complex fftw_complex;
typedef float _Complex fftwf_complex;
#endif

typedef struct hos_hostshim_plan* fftw_plan;
typedef struct hos_hostshim_plan* fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_IN (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)

void fftw_mpi_init(void);
void fftw_mpi_cleanup(void);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0,
                                 ptrdiff_t* local_0_start);
ptrdiff_t fftw_mpi_local_size_2d_transposed(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0,
                                            ptrdiff_t* local_0_start, ptrdiff_t* local_n1,
                                            ptrdiff_t* local_1_start);
double* fftw_alloc_real(size_t n);
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double* in, fftw_complex* out, MPI_Comm comm,
                                   unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, double* out, MPI_Comm comm,
                                   unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* Single-precision names appear only in the driver's branches without
 * USE_DOUBLES; they are declared so that those declarations type-check. */
float* fftwf_alloc_real(size_t n);
fftwf_complex* fftwf_alloc_complex(size_t n);
void fftwf_free(void* p);

#ifdef __cplusplus
}
#endif

#endif
