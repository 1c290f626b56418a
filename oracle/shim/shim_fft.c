/*
 * Single-rank FFTW-MPI / MPI shim implementation for the CPU oracle.
 * TEST INFRASTRUCTURE ONLY: linked with the reference hot-path sources to
 * build oracle/_ref/libhosref_M*.so.  Never linked into the product.
 *
 * Transform definitions (see fftw3-mpi.h for the full statement):
 *   - r2c, TRANSPOSED_OUT, unnormalised: a real-to-complex DFT along y
 *     (exp(-2 pi i ky iy / Ny)) for every x row of the padded real array,
 *     then a complex DFT along x for every ky; written as [Ny/2+1][Nx].
 *   - c2r, TRANSPOSED_IN, unnormalised: a complex inverse DFT along x for
 *     every ky row of the [Ny/2+1][Nx] input, then a complex-to-real inverse
 *     along y that uses only the real parts of the ky=0 and ky=Ny/2 bins.
 *
 * The 1-D kernels are an iterative radix-2 decimation-in-time FFT (Cooley and
 * Tukey 1965) with twiddles from libm cos/sin in double precision, and the
 * standard packing of an n-point real sequence into an n/2-point complex one
 * (e.g. Press et al., Numerical Recipes, sec. 12.3).  Lines are distributed
 * over OpenMP threads.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3-mpi.h"

typedef struct {
  double re, im;
} cpx;

enum { SHIM_R2C = 1, SHIM_C2R = 2 };

struct hos_shim_plan {
  int kind;
  int nx, ny, h; /* h = ny/2 */
  double* real;  /* padded [nx][ny+2] */
  cpx* spec;     /* [h+1][nx] */
  cpx* twx;      /* nx/2 entries exp(-2 pi i k/nx) */
  cpx* twh;      /* h/2 entries exp(-2 pi i k/h) */
  cpx* wy;       /* h+1 entries exp(-2 pi i k/ny) */
  cpx* tmp;      /* [nx][h+1] */
};

static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

static cpx* make_twiddles(int n, int count) {
  cpx* t = (cpx*)malloc(sizeof(cpx) * (size_t)(count > 0 ? count : 1));
  for (int k = 0; k < count; k++) {
    double a = 2.0 * M_PI * (double)k / (double)n;
    t[k].re = cos(a);
    t[k].im = -sin(a);
  }
  return t;
}

/* In-place radix-2 DIT FFT of length n; forward uses exp(-i...), inverse the
 * conjugate; unnormalised. tw holds n/2 forward twiddles for length n. */
static void fft_line(cpx* a, int n, const cpx* tw, int inverse) {
  if (n <= 1) return;
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      cpx t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1, step = n / len;
    for (int i = 0; i < n; i += len) {
      for (int k = 0; k < half; k++) {
        cpx w = tw[k * step];
        if (inverse) w.im = -w.im;
        cpx u = a[i + k];
        cpx x = a[i + k + half];
        cpx v = {x.re * w.re - x.im * w.im, x.re * w.im + x.im * w.re};
        a[i + k].re = u.re + v.re;
        a[i + k].im = u.im + v.im;
        a[i + k + half].re = u.re - v.re;
        a[i + k + half].im = u.im - v.im;
      }
    }
  }
}

/* Real line x[0..ny-1] -> X[0..h], unnormalised forward. */
static void rfft_line(const double* x, cpx* X, const struct hos_shim_plan* p, cpx* work) {
  int h = p->h;
  for (int m = 0; m < h; m++) {
    work[m].re = x[2 * m];
    work[m].im = x[2 * m + 1];
  }
  fft_line(work, h, p->twh, 0);
  for (int k = 0; k <= h; k++) {
    cpx c = work[k % h];
    cpx d = work[(h - k) % h];
    d.im = -d.im; /* conj */
    cpx e = {0.5 * (c.re + d.re), 0.5 * (c.im + d.im)};
    /* o = (c - d) / (2i) = -i (c - d) / 2 */
    cpx o = {0.5 * (c.im - d.im), -0.5 * (c.re - d.re)};
    cpx w = p->wy[k];
    X[k].re = e.re + (w.re * o.re - w.im * o.im);
    X[k].im = e.im + (w.re * o.im + w.im * o.re);
  }
}

/* X[0..h] -> real x[0..ny-1], unnormalised inverse; Im X[0], Im X[h] ignored. */
static void irfft_line(const cpx* Xin, double* x, const struct hos_shim_plan* p, cpx* work) {
  int h = p->h;
  for (int k = 0; k < h; k++) {
    cpx a = Xin[k];
    cpx b = Xin[h - k];
    if (k == 0) {
      a.im = 0.0;
      b.im = 0.0;
    }
    b.im = -b.im; /* conj */
    cpx xe = {a.re + b.re, a.im + b.im};
    cpx df = {a.re - b.re, a.im - b.im};
    /* multiply by exp(+2 pi i k/ny) = conj(wy[k]) */
    cpx w = p->wy[k];
    w.im = -w.im;
    cpx xo = {df.re * w.re - df.im * w.im, df.re * w.im + df.im * w.re};
    /* c = xe + i xo */
    work[k].re = xe.re - xo.im;
    work[k].im = xe.im + xo.re;
  }
  fft_line(work, h, p->twh, 1);
  for (int m = 0; m < h; m++) {
    x[2 * m] = work[m].re;
    x[2 * m + 1] = work[m].im;
  }
}

static struct hos_shim_plan* make_plan(int kind, ptrdiff_t n0, ptrdiff_t n1, double* real, cpx* spec) {
  if (!is_pow2(n0) || !is_pow2(n1) || n0 < 2 || n1 < 4) {
    fprintf(stderr, "oracle shim: sizes must be powers of two (got %td x %td)\n", n0, n1);
    return NULL;
  }
  struct hos_shim_plan* p = (struct hos_shim_plan*)calloc(1, sizeof(*p));
  p->kind = kind;
  p->nx = (int)n0;
  p->ny = (int)n1;
  p->h = (int)(n1 / 2);
  p->real = real;
  p->spec = spec;
  p->twx = make_twiddles(p->nx, p->nx / 2);
  p->twh = make_twiddles(p->h, p->h / 2);
  p->wy = make_twiddles(p->ny, p->h + 1);
  p->tmp = (cpx*)malloc(sizeof(cpx) * (size_t)p->nx * (size_t)(p->h + 1));
  return p;
}

static void exec_r2c(const struct hos_shim_plan* p) {
  int nx = p->nx, ny = p->ny, h = p->h;
  const double* in = p->real;
  cpx* out = p->spec;
  cpx* tmp = p->tmp;
#pragma omp parallel
  {
    cpx* work = (cpx*)malloc(sizeof(cpx) * (size_t)(nx > h + 1 ? nx : h + 1));
#pragma omp for schedule(static)
    for (int ix = 0; ix < nx; ix++) rfft_line(in + (size_t)ix * (size_t)(ny + 2), tmp + (size_t)ix * (size_t)(h + 1), p, work);
#pragma omp for schedule(static)
    for (int ky = 0; ky <= h; ky++) {
      cpx* row = out + (size_t)ky * (size_t)nx;
      for (int ix = 0; ix < nx; ix++) row[ix] = tmp[(size_t)ix * (size_t)(h + 1) + (size_t)ky];
      fft_line(row, nx, p->twx, 0);
    }
    free(work);
  }
}

static void exec_c2r(const struct hos_shim_plan* p) {
  int nx = p->nx, ny = p->ny, h = p->h;
  const cpx* in = p->spec;
  double* out = p->real;
  cpx* tmp = p->tmp;
#pragma omp parallel
  {
    cpx* work = (cpx*)malloc(sizeof(cpx) * (size_t)(nx > h + 1 ? nx : h + 1));
    cpx* col = (cpx*)malloc(sizeof(cpx) * (size_t)(h + 1));
#pragma omp for schedule(static)
    for (int ky = 0; ky <= h; ky++) {
      memcpy(work, in + (size_t)ky * (size_t)nx, sizeof(cpx) * (size_t)nx);
      fft_line(work, nx, p->twx, 1);
      for (int ix = 0; ix < nx; ix++) tmp[(size_t)ix * (size_t)(h + 1) + (size_t)ky] = work[ix];
    }
#pragma omp for schedule(static)
    for (int ix = 0; ix < nx; ix++) {
      memcpy(col, tmp + (size_t)ix * (size_t)(h + 1), sizeof(cpx) * (size_t)(h + 1));
      irfft_line(col, out + (size_t)ix * (size_t)(ny + 2), p, work);
    }
    free(col);
    free(work);
  }
}

void fftw_mpi_init(void) {}

ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0,
                                 ptrdiff_t* local_0_start) {
  (void)comm;
  *local_n0 = n0;
  *local_0_start = 0;
  return n0 * n1;
}

ptrdiff_t fftw_mpi_local_size_2d_transposed(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0,
                                            ptrdiff_t* local_0_start, ptrdiff_t* local_n1,
                                            ptrdiff_t* local_1_start) {
  (void)comm;
  *local_n0 = n0;
  *local_0_start = 0;
  *local_n1 = n1;
  *local_1_start = 0;
  return n0 * n1;
}

double* fftw_alloc_real(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
fftw_complex* fftw_alloc_complex(size_t n) { return (fftw_complex*)calloc(n ? n : 1, sizeof(fftw_complex)); }
void fftw_free(void* p) { free(p); }

fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double* in, fftw_complex* out, MPI_Comm comm,
                                   unsigned flags) {
  (void)comm;
  if (!(flags & FFTW_MPI_TRANSPOSED_OUT)) {
    fprintf(stderr, "oracle shim: only TRANSPOSED_OUT r2c plans are supported\n");
    return NULL;
  }
  return make_plan(SHIM_R2C, n0, n1, in, (cpx*)out);
}

fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, double* out, MPI_Comm comm,
                                   unsigned flags) {
  (void)comm;
  if (!(flags & FFTW_MPI_TRANSPOSED_IN)) {
    fprintf(stderr, "oracle shim: only TRANSPOSED_IN c2r plans are supported\n");
    return NULL;
  }
  return make_plan(SHIM_C2R, n0, n1, out, (cpx*)in);
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (p->kind == SHIM_R2C)
    exec_r2c(p);
  else
    exec_c2r(p);
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  free(p->twx);
  free(p->twh);
  free(p->wy);
  free(p->tmp);
  free(p);
}

float* fftwf_alloc_real(size_t n) { return (float*)calloc(n ? n : 1, sizeof(float)); }
fftwf_complex* fftwf_alloc_complex(size_t n) { return (fftwf_complex*)calloc(n ? n : 1, sizeof(fftwf_complex)); }
void fftwf_free(void* p) { free(p); }
void fftwf_execute(const fftwf_plan p) { (void)p; }

/* ---- MPI, one rank ---- */
int MPI_Init(int* argc, char*** argv) {
  (void)argc;
  (void)argv;
  return 0;
}
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm comm, int* size) {
  (void)comm;
  *size = 1;
  return 0;
}
int MPI_Comm_rank(MPI_Comm comm, int* rank) {
  (void)comm;
  *rank = 0;
  return 0;
}
int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  return 0;
}
/* With one rank a reduction is a copy of count elements of the named type;
 * time_schemes_par.c:76 passes MPI_FLOAT for a double, so 4 bytes are copied
 * exactly as a real single-rank MPI would.  The reference never reads the
 * result (time_schemes_par.c:88 prints the local value). */
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root,
               MPI_Comm comm) {
  (void)op;
  (void)root;
  (void)comm;
  size_t sz = (type == MPI_DOUBLE) ? sizeof(double) : sizeof(float);
  memcpy(recvbuf, sendbuf, sz * (size_t)count);
  return 0;
}
