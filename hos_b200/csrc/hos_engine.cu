// Host engine of the HOS time-advance library: handle lifetime, device
// buffers, the per-stage pass sequence, CUDA-graph capture of a step, and the
// handle C ABI declared in include/hos_gpu.h.
//
// One RHS evaluation (rhs_hos, hosm_2d_par.c:138-235, with Zvel,
// hosm_2d_par.c:240-445) is issued as
//   xinv  : stage input u + dt*sum b k, i kx / z-derivative multipliers, x-inverse
//   yinv  : y-inverse -> eta, eta_x, eta_y, phi_x, phi_y, d_z^j phi^(1)
//   for n = 1..M-1 (Taylor levels of the W recursion):
//     yfwd  : P_n = -sum_m d_z^(n-m) phi^(m+1) eta^(n-m)/(n-m)!, y-forward
//     xfwd  : x-forward (-> phi^(n+1) hat), then z-derivative multipliers, x-inverse
//     yinv  : y-inverse -> d_z^j phi^(n+1), epilogue W_n
//   yfwd  : RHS assembly in physical space, y-forward (rows ky < my only)
//   xfwd  : x-forward, + Dz phi / - g eta, ramp, dealias, k_s, Hamiltonian,
//           final RK update on the last stage
// Every product the reference forms with Mult (operators_par.c:210-235) is a
// pointwise product of fields that both designs obtain through the same c2r,
// so the restructuring changes only the rounding.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <string>
#include <algorithm>
#include <atomic>
#include <map>
#include <utility>
#include <vector>

#include "hos_gpu.h"
#include "hos_persist.h"
#include "hos_registry.h"
#include "hos_stage.h"

namespace hos {
XInvFn lookup_xinv_64(int mode, int n, int e, bool batch);
XFwdFn lookup_xfwd_64(int mode, int n, int e, bool batch);
YInvFn lookup_yinv_64(int mode, int h, int e, bool batch);
YFwdFn lookup_yfwd_64(int mode, int h, int e, bool batch);
XInvFn lookup_xinv_32(int mode, int n, int e, bool batch);
XFwdFn lookup_xfwd_32(int mode, int n, int e, bool batch);
YInvFn lookup_yinv_32(int mode, int h, int e, bool batch);
YFwdFn lookup_yfwd_32(int mode, int h, int e, bool batch);
XInvFn lookup_xinv(int prec, int mode, int n, int e, bool batch) {
  return prec ? lookup_xinv_32(mode, n, e, batch) : lookup_xinv_64(mode, n, e, batch);
}
XFwdFn lookup_xfwd(int prec, int mode, int n, int e, bool batch) {
  return prec ? lookup_xfwd_32(mode, n, e, batch) : lookup_xfwd_64(mode, n, e, batch);
}
YInvFn lookup_yinv(int prec, int mode, int h, int e, bool batch) {
  return prec ? lookup_yinv_32(mode, h, e, batch) : lookup_yinv_64(mode, h, e, batch);
}
YFwdFn lookup_yfwd(int prec, int mode, int h, int e, bool batch) {
  return prec ? lookup_yfwd_32(mode, h, e, batch) : lookup_yfwd_64(mode, h, e, batch);
}

// ---------------------------------------------------------------- small kernels
__global__ void k_set_int(int* p, int v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *p = v;
}

// Active rows of the packed state: 1 + the largest ky row holding a nonzero
// (or non-finite) value in either field, at least `lo`.
__global__ void k_active_rows(const double2* u, size_t fsz, int nx, int row0, int* act) {
  const int row = row0 + blockIdx.x;
  int any = 0;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    const double2 a = u[(size_t)row * nx + i];
    const double2 b = u[fsz + (size_t)row * nx + i];
    if (a.x != 0.0 || a.y != 0.0 || b.x != 0.0 || b.y != 0.0) any = 1;
  }
  any = __syncthreads_or(any);
  if (any && threadIdx.x == 0) atomicMax(act, row + 1);
}

__global__ void k_nonfinite(const double2* u, size_t n, int* flag) {
  int bad = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 a = u[i];
    if (!isfinite(a.x) || !isfinite(a.y)) bad = 1;
  }
  bad = __syncthreads_or(bad);
  if (bad && threadIdx.x == 0) atomicOr(flag, 1);
}

// ---------------------------------------------------------------- embedded error
// Error estimate of an RK45 step: e = sum_s w_s k_s with w_s = dt (c_s - cs_s),
// the difference between the 4th-order update the reference applies and the
// 5th-order one of the same Dormand-Prince stages (time_schemes_par.c:183-235).
// Each block writes max |e| and max |u| over its part of the packed state.
constexpr int ERR_BLOCKS = 296;
struct RkWeights {
  double w[MAX_STAGES];
};
__global__ void __launch_bounds__(256) k_rk_err(const double2* __restrict__ k, int nst, size_t stride, RkWeights w,
                                                const double2* __restrict__ u, size_t n, double* part) {
  __shared__ double se[256], su[256];
  double me = 0.0, mu = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double ex = 0.0, ey = 0.0;
    for (int s = 0; s < nst; s++) {
      const double2 v = k[(size_t)s * stride + i];
      ex += w.w[s] * v.x;
      ey += w.w[s] * v.y;
    }
    me = fmax(me, sqrt(ex * ex + ey * ey));
    const double2 q = u[i];
    mu = fmax(mu, sqrt(q.x * q.x + q.y * q.y));
  }
  se[threadIdx.x] = me;
  su[threadIdx.x] = mu;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) {
      se[threadIdx.x] = fmax(se[threadIdx.x], se[threadIdx.x + off]);
      su[threadIdx.x] = fmax(su[threadIdx.x], su[threadIdx.x + off]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = se[0];
    part[2 * blockIdx.x + 1] = su[0];
  }
}

// ---------------------------------------------------------------- step end
// The step end (StepEndArgs, step_end_body) is in hos_kernels.cuh.
__global__ void __launch_bounds__(256) k_step_end(const double* ham_part, int nparts, double* tdev, double dt,
                                                  long long* stepdev, double* ham_hist, double* t_hist, int hist_cap,
                                                  long long* bad_step) {
  pdl_enter();
  const StepEndArgs a{ham_part, nparts, tdev, dt, stepdev, ham_hist, t_hist, hist_cap, bad_step, nullptr};
  step_end_body(a, blockDim.x);
}

// One block per ensemble member.
__global__ void __launch_bounds__(256) k_step_end_b(const StepEndArgs* __restrict__ arr) {
  pdl_enter();
  const StepEndArgs& a = arr[blockIdx.x];
  if (a.remaining && *a.remaining == 0) return;  // the member's step budget is spent
  step_end_body(a, blockDim.x);
}

// Elementwise spectral operators on one field [h+1][nx] (operators_par.c):
// 0 Dx (i kx, :20-75), 1 Dy (i ky, :85-120), 2 Dz (|k| or |k| tanh(|k|h), :130-196),
// 3 Dealias (:283-325), 4 Sum (:247-279).
__global__ void k_spec_op(Geo g, int op, const double2* a, const double2* b, double2* out) {
  const size_t n = (size_t)(g.h + 1) * g.nx;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(q / g.nx), i = (int)(q % g.nx);
    const double2 x = a[q];
    double2 r;
    if (op == 0) {
      const double kx = kx_of(g, i);
      r = make_double2(-kx * x.y, kx * x.x);
    } else if (op == 1) {
      const double ky = ky_of(g, row);
      r = make_double2(-ky * x.y, ky * x.x);
    } else if (op == 2) {
      const double kx = kx_of(g, i), ky = ky_of(g, row);
      const double m = dz_mult(g, sqrt(kx * kx + ky * ky), 1);
      r = make_double2(m * x.x, m * x.y);
    } else if (op == 3) {
      r = keep_mode(g, i, row) ? x : make_double2(0.0, 0.0);
    } else {
      const double2 y = b[q];
      r = make_double2(x.x + y.x, x.y + y.y);
    }
    out[q] = r;
  }
}

__global__ void k_mul_real(const double* a, const double* b, double* out, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    out[q] = a[q] * b[q];
}

// Hamiltonian (hosm_2d_par.c:462-523): one partial per ky row, weight 1 for
// ky = 0 and 2 otherwise.
__global__ void __launch_bounds__(256) k_ham_rows(Geo g, const double2* eta, const double2* eta_t, const double2* phi,
                                                  double* part) {
  __shared__ double red[256];
  const int row = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < g.nx; i += blockDim.x) {
    const size_t q = (size_t)row * g.nx + i;
    const double2 e = eta[q], et = eta_t[q], p = phi[q];
    s += g.g * e.x * e.x + g.g * e.y * e.y + p.x * et.x + p.y * et.y;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[row] = (row == 0 ? 1.0 : 2.0) * red[0];
}

__global__ void __launch_bounds__(256) k_sum_parts(const double* part, int n, double* out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

}  // namespace hos

using namespace hos;

// ---------------------------------------------------------------- errors
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

namespace hos {
// Lets other translation units of the library report through hos_last_error().
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace hos

#define HOS_CK(x)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) {                                                                       \
      (void)cudaGetLastError();                                                                    \
      return fail(e_ == cudaErrorMemoryAllocation ? HOS_ERR_NOMEM : HOS_ERR_CUDA, "%s: %s", #x,    \
                  cudaGetErrorString(e_));                                                         \
    }                                                                                              \
  } while (0)

// ---------------------------------------------------------------- plan
namespace {

// Elements per thread of each pass kind (x-inverse, x-forward, y-inverse,
// y-forward); defaults, overridable per handle by the autotuner.
struct ElemChoice {
  int xi = 8, xf = 8, yi = 8, yf = 8;          // elements per thread
  int sxi = 0, sxf = 0, syi = 0, syf = 0;      // lines per block scaled by 2^s
  int opb = 16;                                // z-derivative orders per block of the level x-forward pass (all)
  int ys = 16, sys = -1;                       // E and scale of the stage y-inverse pass (YI_JOBS)
  int fuse = 1;                                // next level's y-forward inside each level's y-inverse
};

// Launch geometry of one pass kind: elements per thread E, lines per block,
// threads, dynamic shared memory and (y-passes) the line pitch.
struct KindCfg {
  int e = 8;
  int lines = 1, threads = 0, lp = 0;
  size_t smem = 0;
};

struct PassCfg {
  XInvFn xinv[2] = {};
  XFwdFn xfwd[3] = {};
  YInvFn yinv[2] = {};
  YFwdFn yfwd[3] = {};
  XInvFn xinv_b[2] = {};  // batched variants (per-field arguments from a device array)
  XFwdFn xfwd_b[3] = {};
  YInvFn yinv_b[2] = {};
  YFwdFn yfwd_b[3] = {};
  ElemChoice ec;
  KindCfg xi, xf, yi, yf;
  KindCfg ys;  // the stage y-inverse pass (YI_JOBS); yi is the level one
  const void* twx = nullptr;  // length nx
  const void* twh = nullptr;  // length ny/2
  const void* twy = nullptr;  // length ny
};



int ilog2i(int n) {
  int r = 0;
  while ((1 << r) < n) r++;
  return r;
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Butcher tables of Setup_TimeScheme (time_schemes_par.c:127-314).
int butcher(int scheme, int* nst, double b[MAX_STAGES][MAX_STAGES], double c[MAX_STAGES]) {
  for (int i = 0; i < MAX_STAGES; i++) {
    c[i] = 0.0;
    for (int j = 0; j < MAX_STAGES; j++) b[i][j] = 0.0;
  }
  switch (scheme) {
    case HOS_RK45DP:
      *nst = 7;
      b[1][0] = 1.0 / 5.0;
      b[2][0] = 3.0 / 40.0;
      b[3][0] = 44.0 / 45.0;
      b[4][0] = 19372.0 / 6561.0;
      b[5][0] = 9017.0 / 3168.0;
      b[6][0] = 35.0 / 384.0;
      b[2][1] = 9.0 / 40.0;
      b[3][1] = -56.0 / 15.0;
      b[4][1] = -25360.0 / 2187.0;
      b[5][1] = -355.0 / 33.0;
      b[6][1] = 0.0;
      b[3][2] = 32.0 / 9.0;
      b[4][2] = 64448.0 / 6561.0;
      b[5][2] = 46732.0 / 5247.0;
      b[6][2] = 500.0 / 1113.0;
      b[4][3] = -212.0 / 729.0;
      b[5][3] = 49.0 / 176.0;
      b[6][3] = 125.0 / 192.0;
      b[5][4] = -5103.0 / 18656.0;
      b[6][4] = -2187.0 / 6784.0;
      b[6][5] = 11.0 / 84.0;
      c[0] = 1951.0 / 21600.0;
      c[1] = 0.0;
      c[2] = 22642.0 / 50085.0;
      c[3] = 451.0 / 720.0;
      c[4] = -12231.0 / 42400.0;
      c[5] = 649.0 / 6300.0;
      c[6] = 1.0 / 60.0;
      return 0;
    case HOS_RK4:
      *nst = 4;
      b[1][0] = 0.5;
      b[2][1] = 0.5;
      b[3][2] = 1.0;
      c[0] = 1.0 / 6.0;
      c[1] = 1.0 / 3.0;
      c[2] = 1.0 / 3.0;
      c[3] = 1.0 / 6.0;
      return 0;
    case HOS_EULER:
      *nst = 1;
      c[0] = 1.0;
      return 0;
    case HOS_MIDPOINT:
      *nst = 2;
      b[1][0] = 0.5;
      c[0] = 0.0;
      c[1] = 1.0;
      return 0;
    case HOS_HEUN:
      *nst = 2;
      b[1][0] = 1.0;
      c[0] = 0.5;
      c[1] = 0.5;
      return 0;
    default:
      return -1;
  }
}

// exp(-2 pi i k / n), k < n, from long double libm, rounded once.
std::vector<double2> twiddle_table(int n) {
  std::vector<double2> t(n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n; k++) {
    const long double a = 2.0L * pi * (long double)k / (long double)n;
    t[k].x = (double)cosl(a);
    t[k].y = (double)-sinl(a);
  }
  return t;
}

constexpr int HIST_CAP = 1 << 16;

}  // namespace

struct hos_ctx {
  hos_params p{};
  int nx = 0, ny = 0, h = 0, M = 0, L = 0, prec = 0;
  Geo geo{};
  int nst = 0;
  double b[MAX_STAGES][MAX_STAGES]{};
  double c[MAX_STAGES]{};
  size_t fsz = 0, psz = 0;
  int nz = 0, nphys = 0;
  // device memory
  double2* u = nullptr;
  double2* k = nullptr;
  void* zbuf = nullptr;
  void* phys = nullptr;
  double2* ustage = nullptr;
  double2* ustg = nullptr;  // stage input of the current RK stage
  double2* zvbuf = nullptr; // Zvel outputs / operator scratch (allocated on first use)
  double* hpart = nullptr;  // Hamiltonian row partials (allocated on first use)
  double* hpart_err = nullptr;  // adaptive-step error partials (allocated on first use)
  double2* zplain = nullptr;
  double* pplain = nullptr;
  void* tw[2][3] = {};  // [precision][nx, ny/2, ny] twiddle tables
  double* tdev = nullptr;
  double* trhs = nullptr;
  double* rdev = nullptr;
  long long* stepdev = nullptr;
  long long* bad_step = nullptr;  // first step with a non-finite energy (-1: none)
  int* actdev = nullptr;
  int* flagdev = nullptr;
  double* ham_part = nullptr;
  int nparts = 0;
  double* ham_hist = nullptr;
  double* t_hist = nullptr;
  long long hist_base = 0;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  double g_dt = 0.0;
  bool g_valid = false;
  PassCfg cfg;    // compute precision
  PassCfg cfg64;  // FP64 passes for the boundary transforms
  int device = 0;

  // physical field indices
  int ETA() const { return 0; }
  int ETAX() const { return 1; }
  int ETAY() const { return 2; }
  int PHIX() const { return 3; }
  int PHIY() const { return 4; }
  // d_z^j phi^(i), i = 1..M, j = 1..M+1-i
  int D(int i, int j) const {
    int off = 5;
    for (int q = 1; q < i; q++) off += M + 1 - q;
    return off + (j - 1);
  }
  // W_n, n = 1..L (W_0 = D(1,1))
  int W(int n) const { return n == 0 ? D(1, 1) : 5 + M * (M + 1) / 2 + (n - 1); }
};

namespace {

int scaled_lines(int base, int scale, int maxl) {
  int l = base;
  if (scale > 0) l <<= scale;
  if (scale < 0) l >>= -scale;
  if (l > maxl) l = maxl;
  if (l < 1) l = 1;
  return l;
}

int x_geometry(int n, int e, size_t cs, int scale, KindCfg* k) {
  const int P = n / e;
  int lines = scaled_lines(128 / P > 0 ? 128 / P : 1, scale, MAX_THREADS / P > 0 ? MAX_THREADS / P : 1);
  if (lines * P < 32) lines = 32 / P;
  k->e = e;
  k->lines = lines;
  k->threads = lines * P;
  k->smem = (size_t)lines * (size_t)n * cs;
  if (k->threads % 32 != 0 || k->threads > MAX_THREADS) return -1;
  return 0;
}

int y_geometry(int h, int nx, int e, size_t cs, int scale, KindCfg* k) {
  const int P = h / e;
  int lines = scaled_lines(MAX_THREADS / P > 0 ? MAX_THREADS / P : 1, scale, MAX_THREADS / P > 0 ? MAX_THREADS / P : 1);
  if (lines > nx) lines = nx;
  k->e = e;
  k->lines = lines;
  k->threads = lines * P;
  const int phase = (int)(128 / cs);
  const int target = lines >= phase ? 1 : phase / lines;
  int lp = h + 1;
  while (lp % phase != target % phase) lp++;
  k->lp = lp;
  k->smem = (size_t)lines * lp * cs;
  return k->threads > MAX_THREADS ? -1 : 0;
}

std::mutex g_attr_mu;  // serialises the kernel attribute updates of concurrent hos_create calls

// Largest supported E not above `want` for a line of length n.
int pick_elems(int prec, int n, int want) {
  for (int e = want; e >= 8; e >>= 1)
    if (elems_valid(prec, n, e)) return e;
  return elems_valid(prec, n, 16) ? 16 : 32;
}

// Defaults: E = 8 for every pass kind measured fastest on B200 at 1024^2 in
// both precisions; overridable through HOS_ELEMS="xi,xf,yi,yf".
ElemChoice default_elems(int prec) {
  ElemChoice ec;
  // lines-per-block scales measured fastest on B200 at 1024^2, M = 5
  if (prec) {
    ec.sxi = 1;
  } else {
    ec.sxi = -1;
    ec.syi = -1;
    ec.syf = -1;
  }
  if (const char* s = getenv("HOS_ELEMS")) {
    int a[4];
    if (sscanf(s, "%d,%d,%d,%d", &a[0], &a[1], &a[2], &a[3]) == 4) {
      ec.xi = a[0];
      ec.xf = a[1];
      ec.yi = a[2];
      ec.yf = a[3];
    }
  }
  return ec;
}

int make_cfg(hos_ctx* c, int prec, const ElemChoice& ec, PassCfg* o) {
  const size_t cs = prec ? sizeof(float2) : sizeof(double2);
  const int exi = pick_elems(prec, c->nx, ec.xi), exf = pick_elems(prec, c->nx, ec.xf);
  const int eyi = pick_elems(prec, c->h, ec.yi), eyf = pick_elems(prec, c->h, ec.yf);
  int eys = pick_elems(prec, c->h, ec.ys);
  // a 256-thread block of the stage y-inverse at 16 elements per thread
  // would hold more lines than the grid has rows: use 8 (small grids only)
  if (eys == 16 && MAX_THREADS / (c->h / 16) > c->nx) eys = pick_elems(prec, c->h, 8);
  for (int m = 0; m < 2; m++) o->xinv[m] = lookup_xinv(prec, m, c->nx, exi);
  for (int m = 0; m < 3; m++) o->xfwd[m] = lookup_xfwd(prec, m, c->nx, exf);
  for (int m = 0; m < 2; m++) o->yinv[m] = lookup_yinv(prec, m, c->h, m == YI_JOBS ? eys : eyi);
  for (int m = 0; m < 3; m++) o->yfwd[m] = lookup_yfwd(prec, m, c->h, eyf);
  for (int m = 0; m < 3; m++)
    if (!o->xfwd[m] || !o->yfwd[m] || (m < 2 && (!o->xinv[m] || !o->yinv[m])))
      return fail(HOS_ERR_ARG, "no kernels for %dx%d (E %d/%d/%d/%d)", c->nx, c->ny, exi, exf, eyi, eyf);
  for (int m = 0; m < 2; m++) o->xinv_b[m] = lookup_xinv(prec, m, c->nx, exi, true);
  for (int m = 0; m < 3; m++) o->xfwd_b[m] = lookup_xfwd(prec, m, c->nx, exf, true);
  for (int m = 0; m < 2; m++) o->yinv_b[m] = lookup_yinv(prec, m, c->h, m == YI_JOBS ? eys : eyi, true);
  for (int m = 0; m < 3; m++) o->yfwd_b[m] = lookup_yfwd(prec, m, c->h, eyf, true);
  o->ec = ec;
  if (x_geometry(c->nx, exi, cs, ec.sxi, &o->xi) || x_geometry(c->nx, exf, cs, ec.sxf, &o->xf) ||
      y_geometry(c->h, c->nx, eyi, cs, ec.syi, &o->yi) || y_geometry(c->h, c->nx, eyf, cs, ec.syf, &o->yf) ||
      y_geometry(c->h, c->nx, eys, cs, ec.sys, &o->ys))
    return fail(HOS_ERR_ARG, "no launch geometry for %dx%d", c->nx, c->ny);
  // The dynamic shared memory limit of a kernel is only ever raised: handles
  // with different shapes (and a handle's compute and boundary passes) share
  // kernel functions, and lowering the limit would break the larger launch.
  auto raise = [](const void* f, size_t smem) -> cudaError_t {
    if (!f) return cudaSuccess;
    cudaFuncAttributes at;
    cudaError_t err = cudaFuncGetAttributes(&at, f);
    if (err != cudaSuccess) return err;
    if ((size_t)at.maxDynamicSharedSizeBytes >= smem) return cudaSuccess;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  };
  {
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (int m = 0; m < 2; m++) HOS_CK(raise((const void*)o->xinv[m], o->xi.smem));
    for (int m = 0; m < 3; m++) HOS_CK(raise((const void*)o->xfwd[m], o->xf.smem));
    for (int m = 0; m < 2; m++) HOS_CK(raise((const void*)o->yinv[m], m == YI_JOBS ? o->ys.smem : o->yi.smem));
    for (int m = 0; m < 3; m++) HOS_CK(raise((const void*)o->yfwd[m], o->yf.smem));
    for (int m = 0; m < 2; m++) HOS_CK(raise((const void*)o->xinv_b[m], o->xi.smem));
    for (int m = 0; m < 3; m++) HOS_CK(raise((const void*)o->xfwd_b[m], o->xf.smem));
    for (int m = 0; m < 2; m++) HOS_CK(raise((const void*)o->yinv_b[m], m == YI_JOBS ? o->ys.smem : o->yi.smem));
    for (int m = 0; m < 3; m++) HOS_CK(raise((const void*)o->yfwd_b[m], o->yf.smem));
  }
  o->twx = c->tw[prec][0];
  o->twh = c->tw[prec][1];
  o->twy = c->tw[prec][2];
  return HOS_OK;
}

inline int xgrid(const hos_ctx* c, const KindCfg& k) { return (c->h + 1 + k.lines - 1) / k.lines; }
inline int ygrid(const hos_ctx* c, const KindCfg& k) { return c->nx / k.lines; }

size_t compute_bytes(const hos_params* p, int nst) {
  const size_t nx = p->nx, ny = p->ny, h = ny / 2;
  const size_t fsz = (h + 1) * nx, psz = nx * ny;
  const int M = p->order, L = M - 1;
  const size_t cs = p->precision ? 8 : 16, rs = p->precision ? 4 : 8;
  size_t b = 0;
  b += 2 * fsz * 16;                                 // u
  b += (size_t)nst * 2 * fsz * 16;                   // k
  b += (size_t)(4 + M) * fsz * cs;                   // Z / V scratch
  b += (size_t)(5 + M * (M + 1) / 2 + L) * psz * rs; // physical fields
  b += 2 * fsz * 16 + fsz * 16 + 2 * psz * 8;        // boundary scratch (FP64)
  b += 2 * fsz * 16;                                 // stage input
  b += (nx + h + ny) * (16 + 8);
  b += 2 * (size_t)HIST_CAP * 8 + 4096 * 8 + 4096;
  return b;
}

// Optional per-pass recorder: an event after every launch, with the pass
// kind and its algorithmic bytes (compulsory reads + writes of that pass).
struct PassLog {
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  std::vector<double> bytes;
  int act_rows = 0;
};

enum PassKind { P_XINV_STAGE, P_YINV_STAGE, P_YFWD_LEVEL, P_XFWD_LEVEL, P_YINV_LEVEL, P_YFWD_RHS, P_XFWD_RHS, P_NKIND };
const char* pass_name(int k) {
  static const char* names[P_NKIND] = {"xinv_stage", "yinv_stage", "yfwd_level", "xfwd_level",
                                       "yinv_level", "yfwd_rhs",   "xfwd_rhs"};
  return (k >= 0 && k < P_NKIND) ? names[k] : "?";
}

void log_pass(hos_ctx* c, PassLog* lg, int kind, double bytes) {
  if (!lg) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, c->st);
  lg->ev.push_back(e);
  lg->kind.push_back(kind);
  lg->bytes.push_back(bytes);
}

// One pass launch of a stage: which kernel, its grid and its arguments.  A
// stage is built as a list of these; one field launches them by value, an
// ensemble gathers the arguments of many fields into device arrays and
// launches each pass once per size class (blockIdx.z = field).
enum LaunchKind { L_XINV, L_XFWD, L_YINV, L_YFWD };
struct PassRec {
  int kind = 0, mode = 0;
  int slot = 0;        // position in the stage, shared by the same pass of every member of an ensemble
  int gx = 1, gy = 1;  // grid (x: rows or x-row groups, y: outputs)
  int log_kind = 0;    // PassKind for the per-pass profile
  double bytes = 0.0;  // algorithmic bytes of the launch
  XInvArgs xi{};
  XFwdArgs xf{};
  YInvArgs yi{};
  YFwdArgs yf{};
};

// Column-strip staging of the y-inverse passes: plain loads and shared
// stores (default; measured 1-3 % faster per step on B200 at 1024^2, the
// level y-inverse 3 %), or cp.async with HOS_STRIP=async in the environment.
bool strip_plain() {
  static const bool on = [] {
    const char* s = getenv("HOS_STRIP");
    return !(s && s[0] == 'a');
  }();
  return on;
}

// Builds one RK stage (or one bare RHS evaluation when rhs_only).
// zvel_out: when set, the stage ends after the W recursion and Zvel's four
// spectral outputs W^(M), W^(M-2), (W^2)^(M), (W^2)^(M-2) (hosm_2d_par.c:240-445)
// are written there (4 consecutive FP64 fields) instead of the RHS.
// act_rows is only used for the byte counts of the profile.
void build_stage(hos_ctx* c, int s, double dt, bool rhs_only, double2* uin, double2* kout, const double* tsrc,
                 const int* rows_dev, double2* zvel_out, int act_rows, std::vector<PassRec>& out) {
  const PassCfg& g = c->cfg;
  const int M = c->M, L = c->L;
  const size_t fsz = c->fsz;
  const size_t cs = c->prec ? sizeof(float2) : sizeof(double2);
  const size_t rs = c->prec ? sizeof(float) : sizeof(double);
  char* zb = reinterpret_cast<char*>(c->zbuf);
  const double act = (double)act_rows;
  const double nxd = (double)c->nx, psz = (double)c->psz, fszd = (double)fsz, my = (double)c->geo.my;

  PassRec r1;
  r1.kind = L_XINV;
  r1.mode = XI_STAGE;
  r1.gx = xgrid(c, g.xi);
  r1.gy = 4 + M;
  XInvArgs& xa = r1.xi;
  xa.geo = c->geo;
  xa.ycount = 4 + M;
  xa.rows = c->h + 1;
  xa.rows_dev = rows_dev;
  xa.u = uin;
  int nk = 0;
  for (int p = 0; p < s; p++) {
    if (c->b[s][p] != 0.0) {
      xa.kp[nk] = c->k + (size_t)p * 2 * fsz;
      xa.coef[nk] = dt * c->b[s][p];
      nk++;
    }
  }
  xa.nk = nk;
  xa.z = c->zbuf;
  xa.ustg = c->ustg;
  xa.tdev = tsrc;
  xa.rdev = c->rdev;
  xa.set_ramp = (s == 0);
  xa.tramp = c->p.tramp;
  xa.rampflg = c->p.rampflg;
  r1.slot = 0;
  r1.log_kind = P_XINV_STAGE;
  r1.bytes = act * nxd * (16.0 * 2 * (1 + nk) + (double)cs * (4 + M));
  out.push_back(r1);

  PassRec r2;
  r2.kind = L_YINV;
  r2.mode = YI_JOBS;
  r2.gx = ygrid(c, g.ys);
  YInvArgs& ya = r2.yi;
  ya.geo = c->geo;
  ya.lp = g.ys.lp;
  ya.z = c->zbuf;
  ya.rows_in = c->h + 1;
  ya.rows_dev = rows_dev;
  ya.phys = c->phys;
  ya.plain_strip = strip_plain();
  int nj = 0;
  ya.jobs[nj++] = YJob{0, 0, c->ETA()};
  ya.jobs[nj++] = YJob{0, 1, c->ETAY()};
  ya.jobs[nj++] = YJob{1, 0, c->ETAX()};
  ya.jobs[nj++] = YJob{2, 1, c->PHIY()};
  ya.jobs[nj++] = YJob{3, 0, c->PHIX()};
  for (int j = 1; j <= M; j++) ya.jobs[nj++] = YJob{4 + j - 1, 0, c->D(1, j)};
  ya.ycount = nj;
  r2.gy = nj;
  r2.slot = 1;
  r2.log_kind = P_YINV_STAGE;
  r2.bytes = act * nxd * (double)cs * (4 + M) + psz * (double)rs * (5 + M);
  out.push_back(r2);

  for (int n = 1; n <= L; n++) {
    const bool fused_in = c->cfg.ec.fuse && n >= 2;  // this level's y-forward ran inside level n-1's y-inverse
    if (!fused_in) {
    PassRec r3;
    r3.kind = L_YFWD;
    r3.mode = YF_LEVEL;
    r3.gx = ygrid(c, g.yf);
    r3.gy = 1;
    YFwdArgs& fa = r3.yf;
    fa.geo = c->geo;
    fa.ycount = 1;
    fa.lp = g.yf.lp;
    fa.phys = c->phys;
    fa.eta = c->ETA();
    fa.nterms = n;
    for (int p = 1; p <= n; p++) fa.t_in[p - 1] = c->D(n - p + 1, p);  // power p: m = n - p
    fa.vout = zb;
    fa.rows_out = c->h + 1;
    r3.slot = 2 + 3 * (n - 1);
    r3.log_kind = P_YFWD_LEVEL;
    r3.bytes = psz * (double)rs * (n + 1) + fszd * (double)cs;
    out.push_back(r3);
    }

    PassRec r4;
    r4.kind = L_XFWD;
    r4.mode = XF_LEVEL;
    r4.gx = xgrid(c, g.xf);
    const int opb = c->cfg.ec.opb > 0 ? c->cfg.ec.opb : 1;
    r4.gy = (M - n + opb - 1) / opb;
    XFwdArgs& xf = r4.xf;
    xf.geo = c->geo;
    xf.ycount = r4.gy;
    xf.ndz = M - n;
    xf.opb = opb;
    xf.rows = c->h + 1;
    xf.vin0 = zb;
    xf.zout = zb + fsz * cs;
    r4.slot = 3 + 3 * (n - 1);
    r4.log_kind = P_XFWD_LEVEL;
    r4.bytes = fszd * (double)cs * (1 + M - n);
    out.push_back(r4);

    PassRec r5;
    r5.kind = L_YINV;
    r5.mode = YI_LEVEL;
    r5.gx = ygrid(c, g.yi);
    YInvArgs& yl = r5.yi;
    yl.geo = c->geo;
    yl.lp = g.yi.lp;
    yl.z = c->zbuf;
    yl.rows_in = c->h + 1;
    yl.phys = c->phys;
    yl.plain_strip = strip_plain();
    int nl = 0;
    for (int j = 1; j <= M - n; j++) yl.jobs[nl++] = YJob{1 + j - 1, 0, c->D(n + 1, j)};
    yl.ycount = nl;
    r5.gy = nl;
    yl.w_out = c->W(n);
    yl.eta = c->ETA();
    yl.w_terms = n;
    for (int p = 1; p <= n; p++) yl.w_in[p - 1] = c->D(n - p + 1, p + 1);  // power p: m = n - p
    yl.store_job0 = 1;
    r5.slot = 4 + 3 * (n - 1);
    r5.log_kind = P_YINV_LEVEL;
    r5.bytes = fszd * (double)cs * (M - n) + psz * (double)rs * (M - n + 1 + n + 1);
    if (c->cfg.ec.fuse && n < L) {
      // the next level's P_(n+1) and its y-forward transform in the job-0 blocks;
      // d_z phi^(n+1) (job 0) then has no other reader and is not stored
      yl.fuse_next = 1;
      yl.nx_terms = n + 1;
      for (int p = 2; p <= n + 1; p++) yl.nx_in[p - 1] = c->D(n + 2 - p, p);
      yl.vout = zb;
      yl.store_job0 = 0;
      r5.bytes += psz * (double)rs * (n - 1) + fszd * (double)cs;
    }
    out.push_back(r5);
  }

  if (zvel_out) {
    PassRec rz;
    rz.kind = L_YFWD;
    rz.mode = YF_RHS;
    rz.gx = ygrid(c, g.yf);
    rz.gy = 4;
    YFwdArgs& zf = rz.yf;
    zf.geo = c->geo;
    zf.ycount = 4;
    zf.lp = g.yf.lp;
    zf.phys = c->phys;
    zf.ex = c->ETAX();
    zf.ey = c->ETAY();
    zf.px = c->PHIX();
    zf.py = c->PHIY();
    zf.L = L;
    for (int n = 0; n <= L; n++) zf.w_idx[n] = c->W(n);
    zf.which_base = 2;
    zf.vout = zb;
    zf.rows_out = c->h + 1;
    rz.slot = 100;
    out.push_back(rz);
    PassRec rx;
    rx.kind = L_XFWD;
    rx.mode = XF_PLAIN;
    rx.gx = xgrid(c, g.xf);
    rx.gy = 4;
    XFwdArgs& xz = rx.xf;
    xz.geo = c->geo;
    xz.ycount = 4;
    xz.rows = c->h + 1;
    xz.vin0 = zb;
    xz.out_spec = zvel_out;
    xz.addk_mask = 1 | (L >= 2 ? 2 : 0);  // W^(1) belongs to W^(M) always and to W^(M-2) when L >= 2
    xz.u_add = uin;
    rx.slot = 101;
    out.push_back(rx);
    return;
  }

  PassRec r6;
  r6.kind = L_YFWD;
  r6.mode = YF_RHS;
  r6.gx = ygrid(c, g.yf);
  r6.gy = 2;
  YFwdArgs& ff = r6.yf;
  ff.geo = c->geo;
  ff.ycount = 2;
  ff.lp = g.yf.lp;
  ff.phys = c->phys;
  ff.ex = c->ETAX();
  ff.ey = c->ETAY();
  ff.px = c->PHIX();
  ff.py = c->PHIY();
  ff.L = L;
  for (int n = 0; n <= L; n++) ff.w_idx[n] = c->W(n);
  ff.vout = zb;
  ff.rows_out = c->geo.my;
  r6.slot = 100;
  r6.log_kind = P_YFWD_RHS;
  r6.bytes = psz * (double)rs * (5 + L) + 2.0 * my * nxd * (double)cs;
  out.push_back(r6);

  PassRec r7;
  r7.kind = L_XFWD;
  r7.mode = XF_RHS;
  r7.gx = xgrid(c, g.xf);
  r7.gy = 2;
  XFwdArgs& xe = r7.xf;
  xe.geo = c->geo;
  xe.ycount = 2;
  xe.rows = c->h + 1;
  xe.rows_dev = rows_dev;
  xe.rows_fft = c->geo.my;
  xe.vin0 = zb;
  xe.vin1 = zb + fsz * cs;
  xe.u = uin;
  xe.ustg = c->ustg;
  xe.kout = kout;
  xe.rdev = c->rdev;
  xe.ham = (!rhs_only && s == 0);
  xe.ham_part = c->ham_part;
  xe.final_update = (!rhs_only && s == c->nst - 1);
  for (int p = 0; p < c->nst; p++) {
    xe.kall[p] = c->k + (size_t)p * 2 * fsz;
    xe.cfin[p] = dt * c->c[p];
  }
  xe.nstage = c->nst;
  // V rows < my in, stage input rows < act, k_s rows < my out; on the last
  // stage also the other k's and the updated u (rows < my)
  double b = 2.0 * my * nxd * (double)cs + act * nxd * 16.0 * 2 + my * nxd * 16.0 * 2;
  if (xe.final_update) b += my * nxd * 16.0 * 2 * (c->nst - 1) + my * nxd * 16.0 * 2;
  r7.slot = 101;
  r7.log_kind = P_XFWD_RHS;
  r7.bytes = b;
  out.push_back(r7);
}

// Programmatic dependent launch of the passes of one field (the kernels
// wait for their predecessor at entry, see pdl_enter): the next pass is
// launched and its blocks placed while the previous one drains, which hides
// the launch gap between the dependent passes of a step.  HOS_PDL=0 in the
// environment launches them with plain stream order instead.
bool pdl_enabled() {
  static const bool on = [] {
    const char* s = getenv("HOS_PDL");
    return !(s && s[0] == '0');
  }();
  return on;
}

template <typename... K, typename... A>
void launch_pdl(void (*kernel)(K...), dim3 grid, unsigned threads, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);  // errors surface at the next check
}

// Launches one pass of one field with its arguments by value.
void launch_single(hos_ctx* c, const PassRec& r) {
  const PassCfg& g = c->cfg;
  const dim3 grid(r.gx, r.gy);
  const XInvArgs* nxi = nullptr;
  const XFwdArgs* nxf = nullptr;
  const YInvArgs* nyi = nullptr;
  const YFwdArgs* nyf = nullptr;
  const void* twx = g.twx;
  const void* twh = g.twh;
  const void* twy = g.twy;
  switch (r.kind) {
    case L_XINV: launch_pdl(g.xinv[r.mode], grid, g.xi.threads, g.xi.smem, c->st, r.xi, nxi, twx); break;
    case L_XFWD: launch_pdl(g.xfwd[r.mode], grid, g.xf.threads, g.xf.smem, c->st, r.xf, nxf, twx); break;
    case L_YINV: {
      const KindCfg& k = r.mode == YI_JOBS ? g.ys : g.yi;
      launch_pdl(g.yinv[r.mode], grid, k.threads, k.smem, c->st, r.yi, nyi, twh, twy);
      break;
    }
    default: launch_pdl(g.yfwd[r.mode], grid, g.yf.threads, g.yf.smem, c->st, r.yf, nyf, twh, twy); break;
  }
}

// Enqueues one RK stage (see build_stage) on the handle's stream.
int enqueue_stage(hos_ctx* c, int s, double dt, bool rhs_only, double2* uin, double2* kout, const double* tsrc,
                  const int* rows_dev, PassLog* lg = nullptr, double2* zvel_out = nullptr) {
  std::vector<PassRec> recs;
  build_stage(c, s, dt, rhs_only, uin, kout, tsrc, rows_dev, zvel_out, lg ? lg->act_rows : 0, recs);
  for (const PassRec& r : recs) {
    launch_single(c, r);
    log_pass(c, lg, r.log_kind, r.bytes);
  }
  return HOS_OK;
}

int enqueue_step(hos_ctx* c, double dt) {
  for (int s = 0; s < c->nst; s++) {
    int rc = enqueue_stage(c, s, dt, false, c->u, c->k + (size_t)s * 2 * c->fsz, c->tdev, c->actdev);
    if (rc) return rc;
  }
  const double* hp = c->ham_part;
  launch_pdl(k_step_end, dim3(1), 256, 0, c->st, hp, c->nparts, c->tdev, dt, c->stepdev, c->ham_hist,
             c->t_hist, (int)HIST_CAP, c->bad_step);
  return HOS_OK;
}

int build_graph(hos_ctx* c, double dt) {
  if (c->g_valid && c->g_dt == dt) return HOS_OK;
  if (c->gexec) {
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  if (c->graph) {
    cudaGraphDestroy(c->graph);
    c->graph = nullptr;
  }
  c->g_valid = false;
  HOS_CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(c, dt);
  cudaGraph_t gr = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->st, &gr);
  if (rc) {
    if (gr) cudaGraphDestroy(gr);
    return rc;
  }
  HOS_CK(e);
  c->graph = gr;
  HOS_CK(cudaGraphInstantiate(&c->gexec, c->graph, 0));
  c->g_dt = dt;
  c->g_valid = true;
  return HOS_OK;
}

// Plain FP64 transforms used at the boundary.
int enqueue_r2c(hos_ctx* c, const double* phys_in, double2* spec_out, int dealias) {
  const PassCfg& g = c->cfg64;
  YFwdArgs fa{};
  fa.geo = c->geo;
  fa.lp = g.yf.lp;
  fa.ycount = 1;
  fa.in_ptr = phys_in;
  fa.vout = c->zplain;
  fa.rows_out = c->h + 1;
  g.yfwd[YF_PLAIN]<<<dim3(ygrid(c, g.yf), 1), g.yf.threads, g.yf.smem, c->st>>>(fa, nullptr, g.twh, g.twy);
  XFwdArgs xf{};
  xf.geo = c->geo;
  xf.rows = c->h + 1;
  xf.ycount = 1;
  xf.vin0 = c->zplain;
  xf.out_spec = spec_out;
  xf.dealias = dealias;
  g.xfwd[XF_PLAIN]<<<dim3(xgrid(c, g.xf), 1), g.xf.threads, g.xf.smem, c->st>>>(xf, nullptr, g.twx);
  return HOS_OK;
}

int enqueue_c2r(hos_ctx* c, const double2* spec_in, double* phys_out) {
  const PassCfg& g = c->cfg64;
  XInvArgs xa{};
  xa.geo = c->geo;
  xa.rows = c->h + 1;
  xa.ycount = 1;
  xa.u = spec_in;
  xa.z = c->zplain;
  g.xinv[XI_PLAIN]<<<dim3(xgrid(c, g.xi), 1), g.xi.threads, g.xi.smem, c->st>>>(xa, nullptr, g.twx);
  YInvArgs ya{};
  ya.geo = c->geo;
  ya.lp = g.ys.lp;
  ya.z = c->zplain;
  ya.rows_in = c->h + 1;
  ya.phys = phys_out;
  ya.jobs[0] = YJob{0, 0, 0};
  ya.ycount = 1;
  g.yinv[YI_JOBS]<<<dim3(ygrid(c, g.ys), 1), g.ys.threads, g.ys.smem, c->st>>>(ya, nullptr, g.twh, g.twy);
  return HOS_OK;
}

int refresh_active_rows(hos_ctx* c, const double2* u, int* act) {
  k_set_int<<<1, 32, 0, c->st>>>(act, c->geo.my);
  const int from = c->geo.my;
  if (from < c->h + 1) k_active_rows<<<c->h + 1 - from, 128, 0, c->st>>>(u, c->fsz, c->nx, from, act);
  return HOS_OK;
}

void release(hos_ctx* c) {
  if (!c) return;
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  void* ptrs[] = {c->bad_step, c->u,    c->k,    c->zbuf,    c->phys,   c->ustage, c->ustg, c->zplain,   c->pplain,
                  c->tdev, c->trhs, c->rdev,    c->stepdev, c->actdev, c->flagdev, c->ham_part,
                  c->ham_hist, c->t_hist, c->zvbuf, c->hpart, c->hpart_err, c->tw[0][0], c->tw[0][1], c->tw[0][2], c->tw[1][0], c->tw[1][1], c->tw[1][2]};
  // the handle's memory came from the stream-ordered pool on its stream
  // (dalloc_on): freeing it there waits for nothing else on the device
  for (void* p : ptrs)
    if (p) {
      if (c->st)
        cudaFreeAsync(p, c->st);
      else
        cudaFree(p);
    }
  if (c->st) cudaStreamDestroy(c->st);  // released once its queued frees have run
  delete c;
}

// Fault injection for tests: after `limit` further device allocations, the
// next ones fail as if the device were out of memory.  The limit comes from
// HOS_FAIL_ALLOC_AFTER in the environment or from hos_inject_alloc_failure;
// -1 (the default) disables it.
std::atomic<long> g_alloc_count{0};
std::atomic<long> g_alloc_limit{-2};  // -2: not yet read from the environment

bool injected_alloc_failure() {
  long lim = g_alloc_limit.load();
  if (lim == -2) {
    const char* s = getenv("HOS_FAIL_ALLOC_AFTER");
    long expect = -2;
    g_alloc_limit.compare_exchange_strong(expect, s ? atol(s) : -1L);
    lim = g_alloc_limit.load();
  }
  return lim >= 0 && g_alloc_count.fetch_add(1) >= lim;
}

template <typename P>
int dalloc(P** p, size_t bytes) {
  if (injected_alloc_failure()) {
    *p = nullptr;
    return fail(HOS_ERR_NOMEM, "cudaMalloc(%zu): injected failure (HOS_FAIL_ALLOC_AFTER)", bytes);
  }
  cudaError_t e = cudaMalloc((void**)p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? HOS_ERR_NOMEM : HOS_ERR_CUDA, "cudaMalloc(%zu): %s", bytes,
                cudaGetErrorString(e));
  }
  return HOS_OK;
}

// Bytes the device's stream-ordered pool may keep for reuse after handles
// release memory (HOS_POOL_KEEP_MB, default 8 GiB); above that, released
// memory goes back to the driver at the next synchronisation.
unsigned long long pool_keep_bytes() {
  static const unsigned long long keep = [] {
    const char* s = getenv("HOS_POOL_KEEP_MB");
    return (s && *s) ? (unsigned long long)atoll(s) << 20 : 8ull << 30;
  }();
  return keep;
}

// Sets the release threshold of the current device's default pool once.
void pool_setup() {
  static std::mutex mu;
  static std::vector<int> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (std::find(done.begin(), done.end(), dev) != done.end()) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long keep = pool_keep_bytes();  // the attribute is a 64-bit unsigned value
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  (void)cudaGetLastError();
  done.push_back(dev);
}

// A handle's device memory: from the device's stream-ordered pool, ordered
// on the handle's stream.  Releasing a handle then does not wait for the
// whole device (cudaFree does), and a handle created next reuses the memory
// without going to the driver.  Work on other streams may use the memory
// once the handle's stream has been synchronised.
template <typename P>
int dalloc_on(P** p, size_t bytes, cudaStream_t st) {
  if (injected_alloc_failure()) {
    *p = nullptr;
    return fail(HOS_ERR_NOMEM, "cudaMallocAsync(%zu): injected failure (HOS_FAIL_ALLOC_AFTER)", bytes);
  }
  cudaError_t e = cudaMallocAsync((void**)p, bytes ? bytes : 16, st);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? HOS_ERR_NOMEM : HOS_ERR_CUDA, "cudaMallocAsync(%zu): %s", bytes,
                cudaGetErrorString(e));
  }
  return HOS_OK;
}


// ---------------------------------------------------------------- ensembles
// Fields of one size class (same grid, precision, scheme and kernel shapes)
// advance together: every pass is one launch whose blockIdx.z selects the
// member, with the member's arguments read from a device array.  Classes run
// on their own streams, forked from and joined to the ensemble's stream; a
// whole RK step of all classes is one CUDA graph.
struct EnsClass {
  std::vector<int> idx;  // members
  cudaStream_t st = nullptr;
  cudaEvent_t join = nullptr;
};

}  // namespace

struct hos_ens {
  std::vector<hos_ctx*> mem;
  std::vector<double> dt;
  std::vector<EnsClass> cls;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr;
  void* dargs = nullptr;
  size_t dargs_bytes = 0;
  int* any_bad = nullptr;  // set by a member's step end when its energy is not finite
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int launches_per_step = 0;
  // persistent mode (HOS_ENS_PERSISTENT): one launch of k_persist per step
  int mode = 0;
  PersistArgs pa{};
  void* pbuf = nullptr;  // counters, task list, item list, argument blob
  int pblocks = 0;
  size_t psmem = 0;
  int ntasks = 0;
  int withhold = 0;      // test hook: one task waits for an item that never exists
  int minb = 2;          // resident blocks per SM the persistent kernel is compiled for
  int* rem_cls = nullptr;  // classes mode: per-member step budgets (-1: none)
};

namespace {

bool same_class(const hos_ctx* a, const hos_ctx* b) {
  return a->nx == b->nx && a->ny == b->ny && a->prec == b->prec && a->p.scheme == b->p.scheme &&
         a->cfg.ec.xi == b->cfg.ec.xi && a->cfg.ec.xf == b->cfg.ec.xf && a->cfg.ec.yi == b->cfg.ec.yi &&
         a->cfg.ec.yf == b->cfg.ec.yf && a->cfg.ec.sxi == b->cfg.ec.sxi && a->cfg.ec.sxf == b->cfg.ec.sxf &&
         a->cfg.ec.syi == b->cfg.ec.syi && a->cfg.ec.syf == b->cfg.ec.syf && a->cfg.ec.opb == b->cfg.ec.opb && a->cfg.ec.fuse == b->cfg.ec.fuse &&
         a->cfg.ec.ys == b->cfg.ec.ys && a->cfg.ec.sys == b->cfg.ec.sys &&
         a->device == b->device;
}

struct BatchLaunch {
  int kind, mode, gx, gy, gz;
  size_t off;  // byte offset of the argument array in the device buffer
};

// Builds the launches of one RK step of an ensemble and the host image of
// their argument arrays.
int plan_step(hos_ens* E, std::vector<std::vector<BatchLaunch>>& per_class, std::vector<unsigned char>& img,
              std::vector<StepEndArgs>& ends, std::vector<size_t>& end_off) {
  per_class.assign(E->cls.size(), {});
  auto put = [&](const void* p, size_t n) {
    size_t off = (img.size() + 255) & ~(size_t)255;
    img.resize(off + n);
    std::memcpy(img.data() + off, p, n);
    return off;
  };
  for (size_t ci = 0; ci < E->cls.size(); ci++) {
    const EnsClass& K = E->cls[ci];
    const int nst = E->mem[K.idx[0]]->nst;
    for (int s = 0; s < nst; s++) {
      std::map<int, std::vector<PassRec>> bys;  // slot -> the members' records, in slot order
      for (int f : K.idx) {
        hos_ctx* c = E->mem[f];
        std::vector<PassRec> recs;
        build_stage(c, s, E->dt[f], false, c->u, c->k + (size_t)s * 2 * c->fsz, c->tdev, c->actdev, nullptr, 0, recs);
        for (PassRec& r : recs) {
          r.xi.remaining = r.xf.remaining = r.yi.remaining = r.yf.remaining = E->rem_cls + f;
          bys[r.slot].push_back(r);
        }
      }
      for (const auto& kv : bys) {
        const std::vector<PassRec>& v = kv.second;
        if (v.empty()) continue;
        for (const PassRec& r : v)  // one launch runs one kernel: every record must be of that kernel
          if (r.kind != v[0].kind || r.mode != v[0].mode || r.gx != v[0].gx)
            return fail(HOS_ERR_STATE, "ensemble plan: members disagree at pass slot %d", kv.first);
        BatchLaunch b;
        b.kind = v[0].kind;
        b.mode = v[0].mode;
        b.gx = v[0].gx;
        b.gy = 0;
        b.gz = (int)v.size();
        for (const PassRec& r : v) b.gy = std::max(b.gy, r.gy);
        if (b.kind == L_XINV) {
          std::vector<XInvArgs> a;
          for (const PassRec& r : v) a.push_back(r.xi);
          b.off = put(a.data(), a.size() * sizeof(XInvArgs));
        } else if (b.kind == L_XFWD) {
          std::vector<XFwdArgs> a;
          for (const PassRec& r : v) a.push_back(r.xf);
          b.off = put(a.data(), a.size() * sizeof(XFwdArgs));
        } else if (b.kind == L_YINV) {
          std::vector<YInvArgs> a;
          for (const PassRec& r : v) a.push_back(r.yi);
          b.off = put(a.data(), a.size() * sizeof(YInvArgs));
        } else {
          std::vector<YFwdArgs> a;
          for (const PassRec& r : v) a.push_back(r.yf);
          b.off = put(a.data(), a.size() * sizeof(YFwdArgs));
        }
        per_class[ci].push_back(b);
      }
    }
    std::vector<StepEndArgs> se;
    for (int f : K.idx) {
      hos_ctx* c = E->mem[f];
      se.push_back(StepEndArgs{c->ham_part, c->nparts, c->tdev, E->dt[f], c->stepdev, c->ham_hist,
                               c->t_hist, HIST_CAP, c->bad_step, E->any_bad, E->rem_cls + f});
    }
    end_off.push_back(put(se.data(), se.size() * sizeof(StepEndArgs)));
    ends.insert(ends.end(), se.begin(), se.end());
  }
  return HOS_OK;
}

int build_ens_graph(hos_ens* E) {
  std::vector<std::vector<BatchLaunch>> per_class;
  std::vector<unsigned char> img;
  std::vector<StepEndArgs> ends;
  std::vector<size_t> end_off;
  int prc = plan_step(E, per_class, img, ends, end_off);
  if (prc) return prc;
  if (img.size() > E->dargs_bytes) {
    if (E->dargs) cudaFree(E->dargs);
    E->dargs = nullptr;
    E->dargs_bytes = 0;
    int rc = dalloc(&E->dargs, img.size());
    if (rc) return rc;
    E->dargs_bytes = img.size();
  }
  HOS_CK(cudaMemcpy(E->dargs, img.data(), img.size(), cudaMemcpyHostToDevice));
  if (E->gexec) cudaGraphExecDestroy(E->gexec);
  if (E->graph) cudaGraphDestroy(E->graph);
  E->gexec = nullptr;
  E->graph = nullptr;
  E->launches_per_step = 0;
  HOS_CK(cudaStreamBeginCapture(E->st, cudaStreamCaptureModeThreadLocal));
  cudaEventRecord(E->fork, E->st);
  char* base = reinterpret_cast<char*>(E->dargs);
  for (size_t ci = 0; ci < E->cls.size(); ci++) {
    const EnsClass& K = E->cls[ci];
    const PassCfg& g = E->mem[K.idx[0]]->cfg;
    cudaStreamWaitEvent(K.st, E->fork, 0);
    for (const BatchLaunch& b : per_class[ci]) {
      const dim3 grid(b.gx, b.gy, b.gz);
      void* a = base + b.off;
      switch (b.kind) {
        case L_XINV:
          g.xinv_b[b.mode]<<<grid, g.xi.threads, g.xi.smem, K.st>>>(XInvArgs{}, (const XInvArgs*)a, g.twx);
          break;
        case L_XFWD:
          g.xfwd_b[b.mode]<<<grid, g.xf.threads, g.xf.smem, K.st>>>(XFwdArgs{}, (const XFwdArgs*)a, g.twx);
          break;
        case L_YINV:
          g.yinv_b[b.mode]<<<grid, b.mode == YI_JOBS ? g.ys.threads : g.yi.threads,
                             b.mode == YI_JOBS ? g.ys.smem : g.yi.smem, K.st>>>(YInvArgs{}, (const YInvArgs*)a, g.twh,
                                                                                  g.twy);
          break;
        default:
          g.yfwd_b[b.mode]<<<grid, g.yf.threads, g.yf.smem, K.st>>>(YFwdArgs{}, (const YFwdArgs*)a, g.twh, g.twy);
          break;
      }
      E->launches_per_step++;
    }
    k_step_end_b<<<(unsigned)K.idx.size(), 256, 0, K.st>>>((const StepEndArgs*)(base + end_off[ci]));
    E->launches_per_step++;
    cudaEventRecord(K.join, K.st);
    cudaStreamWaitEvent(E->st, K.join, 0);
  }
  cudaGraph_t gr = nullptr;
  cudaError_t err = cudaStreamEndCapture(E->st, &gr);
  HOS_CK(err);
  E->graph = gr;
  HOS_CK(cudaGraphInstantiate(&E->gexec, E->graph, 0));
  return HOS_OK;
}

// ---------------------------------------------------------------- persistent plan
// The tasks of one RK step of every member (hos_persist.h): the passes
// build_stage gives for each stage, re-shaped for PERSIST_THREADS threads,
// then the step end.  Work items are dealt round by round over the members.
// Blocks per work item.  The members' current tasks together should offer
// about twice as many items as there are resident blocks: a task gets
// ceil(2 * resident / members) items (at least 1), so one field alone spreads
// each pass over the whole GPU and many fields take few, larger items each
// (fewer atomics).  An item holds at most 8 blocks, so that the chain of a
// member's ~50 dependent tasks stays short.
constexpr int PERSIST_MAX_PER_ITEM = 8;

int size_index(int n, int base) {
  for (int s = 0; s < PERSIST_SIZES; s++)
    if (n == (base << s)) return s;
  return -1;
}

int plan_persist(hos_ens* E) {
  struct TaskImg {
    PTask t;
    size_t arg_off;
  };
  std::vector<unsigned char> blob;
  auto put = [&](const void* p, size_t n) {
    size_t off = (blob.size() + 255) & ~(size_t)255;
    blob.resize(off + n);
    std::memcpy(blob.data() + off, p, n);
    return off;
  };
  const int nm = (int)E->mem.size();
  int sms = 0;
  HOS_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E->mem[0]->device));
  const int target_items = std::max(1, (2 * 2 * sms + nm - 1) / nm);  // about 2 resident blocks per SM
  int max_per_item = PERSIST_MAX_PER_ITEM;
  if (const char* ev = getenv("HOS_PERSIST_PER_ITEM")) max_per_item = std::max(1, atoi(ev));
  std::vector<std::vector<TaskImg>> per(nm);
  std::vector<long long> member_items(nm, 0);
  size_t smem = 0;
  for (int f = 0; f < nm; f++) {
    hos_ctx* c = E->mem[f];
    const PassCfg& g = c->cfg;
    const int sx = size_index(c->nx, 64), sy = size_index(c->h, 32);
    if (sx < 0 || sy < 0)
      return fail(HOS_ERR_ARG, "persistent ensemble: member %d grid %dx%d outside 64..2048 x 64..2048", f, c->nx, c->ny);
    if (g.xi.e != 8 || g.xf.e != 8 || g.yi.e != 8 || g.yf.e != 8 || (g.ys.e != 8 && g.ys.e != 16))
      return fail(HOS_ERR_ARG, "persistent ensemble: member %d has tuned kernel shapes (default shapes only)", f);
    const size_t cs = c->prec ? sizeof(float2) : sizeof(double2);
    long long dep = 0;
    auto add = [&](int code, int size_idx, int gx, int gy, const void* args, size_t asz, const void* tw0,
                   const void* tw1) {
      TaskImg ti{};
      ti.t.body = code * PERSIST_SIZES + size_idx;
      ti.t.prec = c->prec;
      ti.t.member = f;
      ti.t.gx = gx;
      ti.t.gy = gy;
      const int nb = gx * gy;
      ti.t.per_item = std::max(1, std::min(max_per_item, (nb + target_items - 1) / target_items));
      ti.t.nitems = (nb + ti.t.per_item - 1) / ti.t.per_item;
      ti.t.dep = dep;
      ti.t.tw0 = tw0;
      ti.t.tw1 = tw1;
      ti.arg_off = put(args, asz);
      dep += ti.t.nitems;
      per[f].push_back(ti);
    };
    for (int s = 0; s < c->nst; s++) {
      std::vector<PassRec> recs;
      build_stage(c, s, E->dt[f], false, c->u, c->k + (size_t)s * 2 * c->fsz, c->tdev, c->actdev, nullptr, 0, recs);
      for (PassRec& r : recs) {
        if (r.kind == L_XINV || r.kind == L_XFWD) {
          const int P = c->nx / 8;
          const int lines = PERSIST_THREADS / P;
          const int gx = (c->h + 1 + lines - 1) / lines;
          smem = std::max(smem, (size_t)lines * c->nx * cs);
          if (r.kind == L_XINV)
            add(PC_XINV_STAGE, sx, gx, r.gy, &r.xi, sizeof(XInvArgs), g.twx, nullptr);
          else
            add(r.mode == XF_LEVEL ? PC_XFWD_LEVEL : PC_XFWD_RHS, sx, gx, r.gy, &r.xf, sizeof(XFwdArgs), g.twx,
                nullptr);
        } else {
          const int e = (r.kind == L_YINV && r.mode == YI_JOBS) ? g.ys.e : 8;
          const int P = c->h / e;
          const int G = PERSIST_THREADS / P;
          if (G > c->nx) return fail(HOS_ERR_ARG, "persistent ensemble: member %d grid too small", f);
          const int phase = (int)(128 / cs);
          const int target = G >= phase ? 1 : phase / G;
          int lp = c->h + 1;
          while (lp % phase != target % phase) lp++;
          smem = std::max(smem, (size_t)G * lp * cs);
          if (r.kind == L_YINV) {
            r.yi.lp = lp;
            const int code = r.mode == YI_LEVEL ? PC_YINV_LEVEL : (e == 16 ? PC_YINV_JOBS : PC_YINV_JOBS8);
            add(code, sy, c->nx / G, r.gy, &r.yi, sizeof(YInvArgs), g.twh, g.twy);
          } else {
            r.yf.lp = lp;
            add(r.mode == YF_LEVEL ? PC_YFWD_LEVEL : PC_YFWD_RHS, sy, c->nx / G, r.gy, &r.yf, sizeof(YFwdArgs), g.twh,
                g.twy);
          }
        }
      }
    }
    const StepEndArgs se{c->ham_part, c->nparts, c->tdev, E->dt[f], c->stepdev, c->ham_hist,
                         c->t_hist, HIST_CAP, c->bad_step, E->any_bad};
    add(PC_STEP_END, 0, 1, 1, &se, sizeof(se), nullptr, nullptr);
    member_items[f] = dep;
  }
  if (E->withhold && !per.empty() && per[0].size() > 1) per[0][1].t.dep += 1;  // an item that never completes

  // the global list: task k of every member, then task k + 1, ...; within a
  // round the members go by grid and precision, so that blocks taking
  // consecutive items mostly run the same pass body (instruction cache)
  std::vector<int> order(nm);
  for (int f = 0; f < nm; f++) order[f] = f;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const hos_ctx* a = E->mem[x];
    const hos_ctx* b = E->mem[y];
    if (a->prec != b->prec) return a->prec < b->prec;
    if (a->nx != b->nx) return a->nx < b->nx;
    return a->ny < b->ny;
  });
  std::vector<PTask> tasks;
  std::vector<size_t> arg_off;
  std::vector<int4> item_task;
  size_t kmax = 0;
  for (auto& v : per) kmax = std::max(kmax, v.size());
  for (size_t k = 0; k < kmax; k++)
    for (int f : order) {
      if (k >= per[f].size()) continue;
      PTask t = per[f][k].t;
      t.first_item = (int)item_task.size();
      for (int i = 0; i < t.nitems; i++)
        item_task.push_back(make_int4((int)tasks.size(), f, (int)t.dep, (int)member_items[f]));
      tasks.push_back(t);
      arg_off.push_back(per[f][k].arg_off);
    }
  if (item_task.size() > (size_t)0x7fffffff) return fail(HOS_ERR_ARG, "persistent ensemble: too many work items");
  for (long long mi : member_items)
    if (mi > 0x7fffffffLL) return fail(HOS_ERR_ARG, "persistent ensemble: too many work items in one member's step");

  // one device buffer: counters | done[nm] | member_items[nm] | remaining[nm] | tasks | item_task | argument blob
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t o_cnt = 0, o_done = 256, o_mi = al(o_done + nm * 8), o_rem = al(o_mi + nm * 8);
  const size_t o_tasks = al(o_rem + nm * 4);
  const size_t o_items = al(o_tasks + tasks.size() * sizeof(PTask));
  const size_t o_blob = al(o_items + item_task.size() * sizeof(int4));
  const size_t total = o_blob + blob.size();
  if (E->pbuf) cudaFree(E->pbuf);
  if (E->rem_cls) cudaFree(E->rem_cls);
  E->pbuf = nullptr;
  int rc = dalloc(&E->pbuf, total);
  if (rc) return rc;
  char* base = static_cast<char*>(E->pbuf);
  for (size_t i = 0; i < tasks.size(); i++) tasks[i].args = base + o_blob + arg_off[i];
  std::vector<unsigned char> img(o_blob, 0);
  std::memcpy(img.data() + o_mi, member_items.data(), nm * 8);
  std::memset(img.data() + o_rem, 0xff, nm * 4);  // -1: no step budget
  std::memcpy(img.data() + o_tasks, tasks.data(), tasks.size() * sizeof(PTask));
  std::memcpy(img.data() + o_items, item_task.data(), item_task.size() * sizeof(int4));
  HOS_CK(cudaMemcpy(base, img.data(), img.size(), cudaMemcpyHostToDevice));
  HOS_CK(cudaMemcpy(base + o_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice));

  PersistArgs& a = E->pa;
  a.tasks = reinterpret_cast<const PTask*>(base + o_tasks);
  a.item_info = reinterpret_cast<const int4*>(base + o_items);
  a.nitems = (int)item_task.size();
  a.done = reinterpret_cast<unsigned long long*>(base + o_done);
  a.member_items = reinterpret_cast<const long long*>(base + o_mi);
  a.nmembers = nm;
  a.remaining = reinterpret_cast<int*>(base + o_rem);
  a.head = reinterpret_cast<unsigned int*>(base + o_cnt);
  a.finished = reinterpret_cast<unsigned int*>(base + o_cnt + 4);
  a.epoch = reinterpret_cast<unsigned long long*>(base + o_cnt + 8);
  a.err = reinterpret_cast<int*>(base + o_cnt + 16);
  a.err_info = reinterpret_cast<long long*>(base + o_cnt + 32);
  if (a.wait_limit_ns <= 0) a.wait_limit_ns = 2000000000LL;  // 2 s
  E->ntasks = (int)tasks.size();

  // 3 resident blocks per SM (80 registers a thread) when every grid is at
  // most 256 points per direction, where more warps pay more than the
  // spills of the heavier bodies cost; 2 otherwise.  HOS_PERSIST_MINB=2|3 in
  // the environment overrides.
  int maxn = 0;
  for (hos_ctx* c : E->mem) maxn = std::max(maxn, std::max(c->nx, c->ny));
  E->minb = maxn <= 256 ? 3 : 2;
  if (const char* ev = getenv("HOS_PERSIST_MINB")) E->minb = (ev[0] == '3') ? 3 : 2;
  // resident blocks: the launch is cooperative, so all of them must fit at once
  smem = std::max(smem, (size_t)16);
  HOS_CK(persist_set_smem(smem, E->minb));
  int per_sm = 0;
  HOS_CK(persist_occupancy(&per_sm, smem, E->minb));
  if (per_sm < 1) return fail(HOS_ERR_ARG, "persistent ensemble: kernel does not fit an SM");
  E->pblocks = per_sm * sms;
  E->psmem = smem;
  E->launches_per_step = 1;
  return HOS_OK;
}

void release_ens(hos_ens* E) {
  if (!E) return;
  if (E->pbuf) cudaFree(E->pbuf);
  if (E->gexec) cudaGraphExecDestroy(E->gexec);
  if (E->graph) cudaGraphDestroy(E->graph);
  if (E->dargs) cudaFree(E->dargs);
  if (E->any_bad) cudaFree(E->any_bad);
  for (EnsClass& K : E->cls) {
    if (K.join) cudaEventDestroy(K.join);
    if (K.st) cudaStreamDestroy(K.st);
  }
  if (E->fork) cudaEventDestroy(E->fork);
  if (E->st) cudaStreamDestroy(E->st);
  delete E;
}

}  // namespace

// ---------------------------------------------------------------- C ABI
extern "C" {

void hos_default_params(hos_params* p, int nx, int ny) {
  std::memset(p, 0, sizeof(*p));
  p->nx = nx;
  p->ny = ny;
  p->lx = 2 * M_PI;
  p->ly = 2 * M_PI;
  p->g = 1.0;
  p->order = 3;
  p->precision = HOS_PREC_FP64;
  p->depth = 0.0;
  p->rampflg = 0;
  p->tramp = 1.0;
  p->scheme = HOS_RK4;
  p->mx = 0;
  p->my = 0;
}

const char* hos_last_error(void) { return g_err.c_str(); }

const char* hos_version(void) {
  return "hos_b200 sm_100a: Stockham line FFT passes (radix-8/16), fused HOS RHS, FP64/FP32 compute";
}

size_t hos_footprint_bytes(const hos_params* p) {
  if (!p) return 0;
  int nst = 0;
  double b[MAX_STAGES][MAX_STAGES], c[MAX_STAGES];
  if (butcher(p->scheme, &nst, b, c)) return 0;
  return compute_bytes(p, nst);
}

int hos_device_free_bytes(size_t* free_bytes) {
  if (!free_bytes) return fail(HOS_ERR_ARG, "null argument");
  size_t fr = 0, tot = 0;
  HOS_CK(cudaMemGetInfo(&fr, &tot));
  int dev = 0;
  HOS_CK(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  HOS_CK(cudaDeviceGetDefaultMemPool(&pool, dev));
  unsigned long long reserved = 0, used = 0;
  HOS_CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
  HOS_CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
  *free_bytes = fr + (size_t)(reserved > used ? reserved - used : 0);
  return HOS_OK;
}

int hos_create(const hos_params* p, hos_handle* out) {
  if (!p || !out) return fail(HOS_ERR_ARG, "null argument");
  *out = nullptr;
  if (!pow2(p->nx) || !pow2(p->ny) || p->nx < 16 || p->ny < 16 || p->nx > 4096 || p->ny > 4096)
    return fail(HOS_ERR_ARG, "grid %dx%d: sizes must be powers of two in [16, 4096]", p->nx, p->ny);
  if (p->order < 1 || p->order > 7) return fail(HOS_ERR_ARG, "order M=%d outside 1..7", p->order);
  if (p->precision != HOS_PREC_FP64 && p->precision != HOS_PREC_FP32)
    return fail(HOS_ERR_ARG, "precision %d", p->precision);
  if (!(p->lx > 0) || !(p->ly > 0)) return fail(HOS_ERR_ARG, "domain lengths must be positive");
  if (p->rampflg == 1 && !(p->tramp != 0)) return fail(HOS_ERR_ARG, "ramp with Tramp = 0");
  hos_ctx* c = new hos_ctx();
  c->p = *p;
  c->nx = p->nx;
  c->ny = p->ny;
  c->h = p->ny / 2;
  c->M = p->order;
  c->L = p->order - 1;
  c->prec = p->precision;
  if (butcher(p->scheme, &c->nst, c->b, c->c)) {
    delete c;
    return fail(HOS_ERR_ARG, "unknown scheme %d", p->scheme);
  }
  cudaGetDevice(&c->device);
  Geo& G = c->geo;
  G.nx = c->nx;
  G.ny = c->ny;
  G.h = c->h;
  // operators_par.c:290-291
  G.mx = p->mx > 0 ? p->mx : (int)std::floor(0.5 * c->nx / (1 + 0.5 * c->L));
  G.my = p->my > 0 ? p->my : (int)std::floor(0.5 * c->ny / (1 + 0.5 * c->L));
  if (G.my > c->h + 1) G.my = c->h + 1;
  if (G.my < 1) G.my = 1;
  G.kx0 = 2 * M_PI / p->lx;  // hdf5_routines_2d_par.c:98-99
  G.ky0 = 2 * M_PI / p->ly;
  G.depth = p->depth;
  G.g = p->g;
  G.inv_nxny = 1.0 / ((double)c->nx * (double)c->ny);
  c->fsz = (size_t)(c->h + 1) * c->nx;
  c->psz = (size_t)c->nx * c->ny;
  c->nz = 4 + c->M;
  c->nphys = 5 + c->M * (c->M + 1) / 2 + c->L;
  const size_t cs = c->prec ? sizeof(float2) : sizeof(double2);
  const size_t rs = c->prec ? sizeof(float) : sizeof(double);
  int rc = HOS_OK;
  // The handle's own stream takes the greatest priority: its work (uploads,
  // steps of one field, read-backs) is short, and a server creates and reads
  // fields while an ensemble's long chunk occupies the device.
  int prio_least = 0, prio_greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->st, cudaStreamNonBlocking, prio_greatest);
  if (e != cudaSuccess) {
    delete c;
    return fail(HOS_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  pool_setup();
#define HOS_AL(ptr, bytes)                    \
  do {                                        \
    rc = dalloc_on(&(ptr), (bytes), c->st);   \
    if (rc) {                       \
      release(c);                   \
      return rc;                    \
    }                               \
  } while (0)
  HOS_AL(c->u, 2 * c->fsz * sizeof(double2));
  HOS_AL(c->k, (size_t)c->nst * 2 * c->fsz * sizeof(double2));
  HOS_AL(c->zbuf, (size_t)c->nz * c->fsz * cs);
  HOS_AL(c->phys, (size_t)c->nphys * c->psz * rs);
  HOS_AL(c->ustage, 2 * c->fsz * sizeof(double2));
  HOS_AL(c->ustg, 2 * c->fsz * sizeof(double2));
  HOS_AL(c->zplain, c->fsz * sizeof(double2));
  HOS_AL(c->pplain, 2 * c->psz * sizeof(double));
  {
    const int lens[3] = {c->nx, c->h, c->ny};
    for (int q = 0; q < 3; q++) {
      HOS_AL(c->tw[0][q], (size_t)lens[q] * sizeof(double2));
      HOS_AL(c->tw[1][q], (size_t)lens[q] * sizeof(float2));
    }
  }
  HOS_AL(c->tdev, sizeof(double));
  HOS_AL(c->trhs, sizeof(double));
  HOS_AL(c->rdev, sizeof(double));
  HOS_AL(c->stepdev, sizeof(long long));
  HOS_AL(c->bad_step, sizeof(long long));
  HOS_AL(c->actdev, sizeof(int));
  HOS_AL(c->flagdev, sizeof(int));
  HOS_AL(c->ham_hist, HIST_CAP * sizeof(double));
  HOS_AL(c->t_hist, HIST_CAP * sizeof(double));
#undef HOS_AL
  {
    ElemChoice ec = default_elems(c->prec);
    ElemChoice ec64 = default_elems(0);
    // shapes chosen by the autotuner (hos_params.tune): E per pass kind, then
    // the lines-per-block scale exponents
    if (p->tune[0]) ec.xi = p->tune[0];
    if (p->tune[1]) ec.xf = p->tune[1];
    if (p->tune[2]) ec.yi = p->tune[2];
    if (p->tune[3]) ec.yf = p->tune[3];
    auto clamp3 = [](int v) { return v < -3 ? -3 : (v > 3 ? 3 : v); };
    bool tuned = false;
    for (int i = 0; i < 8; i++) tuned = tuned || p->tune[i] != 0;
    if (tuned) {  // a tuned shape sets every scale (0 included)
      ec.sxi = clamp3(p->tune[4]);
      ec.sxf = clamp3(p->tune[5]);
      ec.syi = clamp3(p->tune[6]);
      ec.syf = clamp3(p->tune[7]);
    }
    if (p->tune_opb > 0) ec.opb = p->tune_opb;
    if (p->tune_ys) {  // the stage y-inverse tuned on its own; otherwise it follows the level one
      ec.ys = p->tune_ys;
      ec.sys = clamp3(p->tune_sys);
    } else if (tuned) {
      ec.ys = ec.yi;
      ec.sys = ec.syi;
    }
    if (p->tune_nofuse) ec.fuse = 0;
    rc = make_cfg(c, c->prec, ec, &c->cfg);
    if (!rc) rc = make_cfg(c, 0, ec64, &c->cfg64);
  }
  if (rc) {
    release(c);
    return rc;
  }
  c->nparts = c->h + 1;  // one Hamiltonian partial per ky row
  rc = dalloc_on(&c->ham_part, (size_t)c->nparts * sizeof(double), c->st);
  if (rc) {
    release(c);
    return rc;
  }
  // twiddles, zeroed state and stage buffers (rows ky >= my of k are never written)
  e = cudaSuccess;
  {
    const int lens[3] = {c->nx, c->h, c->ny};
    for (int q = 0; q < 3 && e == cudaSuccess; q++) {
      std::vector<double2> tw = twiddle_table(lens[q]);
      std::vector<float2> tw32(lens[q]);
      for (int i = 0; i < lens[q]; i++) tw32[i] = make_float2((float)tw[i].x, (float)tw[i].y);
      // on the handle's stream, after its allocations (pageable sources: the
      // copies are staged before the calls return)
      e = cudaMemcpyAsync(c->tw[0][q], tw.data(), lens[q] * sizeof(double2), cudaMemcpyHostToDevice, c->st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->tw[1][q], tw32.data(), lens[q] * sizeof(float2), cudaMemcpyHostToDevice, c->st);
    }
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(c->u, 0, 2 * c->fsz * sizeof(double2), c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->k, 0, (size_t)c->nst * 2 * c->fsz * sizeof(double2), c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->tdev, 0, sizeof(double), c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->trhs, 0, sizeof(double), c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->stepdev, 0, sizeof(long long), c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->bad_step, 0xff, sizeof(long long), c->st);  // -1
  if (e == cudaSuccess) e = cudaMemsetAsync(c->ham_part, 0, (size_t)c->nparts * sizeof(double), c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->ham_hist, 0, HIST_CAP * sizeof(double), c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->t_hist, 0, HIST_CAP * sizeof(double), c->st);
  if (e == cudaSuccess) {
    k_set_int<<<1, 32, 0, c->st>>>(c->actdev, c->geo.my);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) {
    release(c);
    return fail(HOS_ERR_CUDA, "init: %s", cudaGetErrorString(e));
  }
  *out = c;
  return HOS_OK;
}

int hos_destroy(hos_handle h) {
  if (!h) return HOS_OK;
  cudaStreamSynchronize(h->st);
  release(h);
  return HOS_OK;
}

int hos_get_bounds(hos_handle h, int* mx, int* my) {
  if (!h) return fail(HOS_ERR_ARG, "null handle");
  if (mx) *mx = h->geo.mx;
  if (my) *my = h->geo.my;
  return HOS_OK;
}

void* hos_stream(hos_handle h) { return h ? (void*)h->st : nullptr; }

int hos_set_state_spectral(hos_handle h, const double* u, double t) {
  if (!h || !u) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(cudaMemsetAsync(h->bad_step, 0xff, sizeof(long long), h->st));
  HOS_CK(host_copy(h->u, u, 2 * h->fsz * sizeof(double2), h->st));
  HOS_CK(cudaMemcpyAsync(h->tdev, &t, sizeof(double), cudaMemcpyHostToDevice, h->st));
  refresh_active_rows(h, h->u, h->actdev);
  HOS_CK(cudaGetLastError());
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_get_state_spectral(hos_handle h, double* u, double* t) {
  if (!h || !u) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(host_copy(u, h->u, 2 * h->fsz * sizeof(double2), h->st));
  double tt = 0;
  HOS_CK(cudaMemcpyAsync(&tt, h->tdev, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  if (t) *t = tt;
  return HOS_OK;
}

int hos_set_state_physical(hos_handle h, const double* eta, const double* phi, double t) {
  if (!h || !eta || !phi) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(cudaMemsetAsync(h->bad_step, 0xff, sizeof(long long), h->st));
  HOS_CK(host_copy(h->pplain, eta, h->psz * sizeof(double), h->st));
  HOS_CK(host_copy(h->pplain + h->psz, phi, h->psz * sizeof(double), h->st));
  enqueue_r2c(h, h->pplain, h->u, 1);
  enqueue_r2c(h, h->pplain + h->psz, h->u + h->fsz, 1);
  HOS_CK(cudaMemcpyAsync(h->tdev, &t, sizeof(double), cudaMemcpyHostToDevice, h->st));
  refresh_active_rows(h, h->u, h->actdev);
  HOS_CK(cudaGetLastError());
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_get_state_physical(hos_handle h, double* eta, double* phi) {
  if (!h || !eta || !phi) return fail(HOS_ERR_ARG, "null argument");
  enqueue_c2r(h, h->u, h->pplain);
  enqueue_c2r(h, h->u + h->fsz, h->pplain + h->psz);
  HOS_CK(cudaGetLastError());
  HOS_CK(host_copy(eta, h->pplain, h->psz * sizeof(double), h->st));
  HOS_CK(host_copy(phi, h->pplain + h->psz, h->psz * sizeof(double), h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_step(hos_handle h, double dt, int nsteps) {
  if (!h) return fail(HOS_ERR_ARG, "null handle");
  if (nsteps < 0) return fail(HOS_ERR_ARG, "nsteps < 0");
  if (nsteps == 0) return HOS_OK;
  int rc = build_graph(h, dt);
  if (rc) return rc;
  for (int i = 0; i < nsteps; i++) HOS_CK(cudaGraphLaunch(h->gexec, h->st));
  return HOS_OK;
}

int hos_step_adaptive(hos_handle h, double t_end, double* dt, double rtol, double atol, int max_steps,
                      int* accepted, int* rejected) {
  if (!h || !dt) return fail(HOS_ERR_ARG, "null argument");
  if (h->p.scheme != HOS_RK45DP) return fail(HOS_ERR_STATE, "adaptive steps need the RK45 scheme (scheme 1)");
  if (!(*dt > 0.0) || !(rtol >= 0.0) || !(atol >= 0.0) || (rtol == 0.0 && atol == 0.0) || max_steps < 1)
    return fail(HOS_ERR_ARG, "bad dt, tolerances or step limit");
  // 5th-order weights of the pair (time_schemes_par.c:225-231); the update uses c (4th order), as the reference does
  static const double cs[7] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
  if (!h->hpart_err) {
    int rc = dalloc_on(&h->hpart_err, (size_t)2 * ERR_BLOCKS * sizeof(double), h->st);
    if (rc) return rc;
  }
  int acc = 0, rej = 0;
  double t = 0.0;
  long long step0 = 0;
  HOS_CK(cudaMemcpyAsync(&t, h->tdev, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  std::vector<double> part(2 * ERR_BLOCKS);
  const double span = std::max(std::fabs(t_end), std::fabs(t));
  double dtry = *dt;
  while (t_end - t > 1e-12 * span && acc + rej < max_steps) {
    const double dts = std::min(dtry, t_end - t);
    HOS_CK(cudaMemcpyAsync(&step0, h->stepdev, sizeof(long long), cudaMemcpyDeviceToHost, h->st));
    HOS_CK(cudaMemcpyAsync(h->ustage, h->u, 2 * h->fsz * sizeof(double2), cudaMemcpyDeviceToDevice, h->st));
    int rc = enqueue_step(h, dts);
    if (rc) return rc;
    RkWeights w{};
    for (int s = 0; s < h->nst; s++) w.w[s] = dts * (h->c[s] - cs[s]);
    k_rk_err<<<ERR_BLOCKS, 256, 0, h->st>>>(h->k, h->nst, 2 * h->fsz, w, h->u, 2 * h->fsz, h->hpart_err);
    HOS_CK(cudaGetLastError());
    HOS_CK(cudaMemcpyAsync(part.data(), h->hpart_err, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    HOS_CK(cudaStreamSynchronize(h->st));
    double me = 0.0, mu = 0.0;
    for (int b = 0; b < ERR_BLOCKS; b++) {
      me = std::max(me, part[2 * b]);
      mu = std::max(mu, part[2 * b + 1]);
    }
    const double err = me / (atol + rtol * mu);
    if (!std::isfinite(err)) return fail(HOS_ERR_NONFINITE, "adaptive step at t=%g: error estimate not finite", t);
    if (err <= 1.0) {
      acc++;
      t += dts;
    } else {  // rejected: the state, time and step count go back to the step's start
      rej++;
      HOS_CK(cudaMemcpyAsync(h->u, h->ustage, 2 * h->fsz * sizeof(double2), cudaMemcpyDeviceToDevice, h->st));
      HOS_CK(cudaMemcpyAsync(h->tdev, &t, sizeof(double), cudaMemcpyHostToDevice, h->st));
      HOS_CK(cudaMemcpyAsync(h->stepdev, &step0, sizeof(long long), cudaMemcpyHostToDevice, h->st));
      HOS_CK(cudaStreamSynchronize(h->st));
    }
    // elementary controller for a 4th/5th-order pair: safety 0.9, growth in [0.2, 5]
    const double fac = err == 0.0 ? 5.0 : std::min(5.0, std::max(0.2, 0.9 * std::pow(err, -0.2)));
    dtry = dts * fac;
  }
  // the time the host tracked is the device's to the last rounding: keep the device's
  *dt = dtry;
  if (accepted) *accepted = acc;
  if (rejected) *rejected = rej;
  if (t_end - t > 1e-12 * span) return fail(HOS_ERR_STATE, "adaptive steps stopped at t=%g after %d attempts", t, acc + rej);
  return HOS_OK;
}

int hos_sync(hos_handle h) {
  if (!h) return fail(HOS_ERR_ARG, "null handle");
  HOS_CK(cudaStreamSynchronize(h->st));
  HOS_CK(cudaGetLastError());
  long long bad = -1;
  HOS_CK(cudaMemcpy(&bad, h->bad_step, sizeof(long long), cudaMemcpyDeviceToHost));
  if (bad >= 0) return fail(HOS_ERR_NONFINITE, "the state became non-finite at step %lld", bad);
  return HOS_OK;
}

void hos_inject_alloc_failure(long after) {
  g_alloc_count.store(0);
  g_alloc_limit.store(after < 0 ? -1 : after);
}

int hos_health(hos_handle h, long long* first_nonfinite_step) {
  if (!h || !first_nonfinite_step) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(cudaStreamSynchronize(h->st));
  HOS_CK(cudaMemcpy(first_nonfinite_step, h->bad_step, sizeof(long long), cudaMemcpyDeviceToHost));
  return HOS_OK;
}

int hos_energy_history(hos_handle h, double* t_out, double* ham_out, int max, int* count) {
  if (!h || !count) return fail(HOS_ERR_ARG, "null argument");
  long long steps = 0;
  HOS_CK(cudaMemcpyAsync(&steps, h->stepdev, sizeof(long long), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  long long first = h->hist_base;
  if (steps - first > HIST_CAP) first = steps - HIST_CAP;
  long long n = steps - first;
  if (n > max) {
    first = steps - max;
    n = max;
  }
  // the n records are consecutive slots of the ring (at most two runs);
  // only those are read back
  std::vector<double> th((size_t)n), hh((size_t)n);
  for (long long i = 0; i < n;) {
    const long long slot = (first + i) % HIST_CAP;
    const long long run = std::min(n - i, (long long)HIST_CAP - slot);
    HOS_CK(cudaMemcpyAsync(th.data() + i, h->t_hist + slot, (size_t)run * sizeof(double), cudaMemcpyDeviceToHost,
                           h->st));
    HOS_CK(cudaMemcpyAsync(hh.data() + i, h->ham_hist + slot, (size_t)run * sizeof(double), cudaMemcpyDeviceToHost,
                           h->st));
    i += run;
  }
  if (n > 0) HOS_CK(cudaStreamSynchronize(h->st));
  for (long long i = 0; i < n; i++) {
    if (t_out) t_out[i] = th[(size_t)i];
    if (ham_out) ham_out[i] = hh[(size_t)i];
  }
  *count = (int)n;
  return HOS_OK;
}

int hos_clear_history(hos_handle h) {
  if (!h) return fail(HOS_ERR_ARG, "null handle");
  long long steps = 0;
  HOS_CK(cudaMemcpyAsync(&steps, h->stepdev, sizeof(long long), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  h->hist_base = steps;
  return HOS_OK;
}

int hos_rhs(hos_handle h, const double* u, double* rhs, double t) {
  if (!h || !u || !rhs) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(host_copy(h->ustage, u, 2 * h->fsz * sizeof(double2), h->st));
  HOS_CK(cudaMemcpyAsync(h->trhs, &t, sizeof(double), cudaMemcpyHostToDevice, h->st));
  // the last stage buffer is scratch between steps; rows ky >= my stay zero
  double2* kout = h->k + (size_t)(h->nst - 1) * 2 * h->fsz;
  int rc = enqueue_stage(h, 0, 0.0, true, h->ustage, kout, h->trhs, nullptr);
  if (rc) return rc;
  HOS_CK(cudaGetLastError());
  HOS_CK(host_copy(rhs, kout, 2 * h->fsz * sizeof(double2), h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_fft_2d_ld(hos_handle h, const double* u_phys, int ld, double* hu) {
  if (!h || !u_phys || !hu || ld < h->ny) return fail(HOS_ERR_ARG, "bad argument");
  HOS_CK(cudaMemcpy2DAsync(h->pplain, h->ny * sizeof(double), u_phys, (size_t)ld * sizeof(double),
                           h->ny * sizeof(double), h->nx, cudaMemcpyDefault, h->st));
  enqueue_r2c(h, h->pplain, h->ustage, 0);
  HOS_CK(cudaGetLastError());
  HOS_CK(host_copy(hu, h->ustage, h->fsz * sizeof(double2), h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_ifft_2d_ld(hos_handle h, const double* hu, double* u_phys, int ld) {
  if (!h || !hu || !u_phys || ld < h->ny) return fail(HOS_ERR_ARG, "bad argument");
  HOS_CK(host_copy(h->ustage, hu, h->fsz * sizeof(double2), h->st));
  enqueue_c2r(h, h->ustage, h->pplain);
  HOS_CK(cudaGetLastError());
  HOS_CK(cudaMemcpy2DAsync(u_phys, (size_t)ld * sizeof(double), h->pplain, h->ny * sizeof(double),
                           h->ny * sizeof(double), h->nx, cudaMemcpyDefault, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_fft_2d(hos_handle h, const double* u_phys, double* hu) {
  if (!h || !u_phys || !hu) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(host_copy(h->pplain, u_phys, h->psz * sizeof(double), h->st));
  enqueue_r2c(h, h->pplain, h->ustage, 0);
  HOS_CK(cudaGetLastError());
  HOS_CK(host_copy(hu, h->ustage, h->fsz * sizeof(double2), h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_ifft_2d(hos_handle h, const double* hu, double* u_phys) {
  if (!h || !hu || !u_phys) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(host_copy(h->ustage, hu, h->fsz * sizeof(double2), h->st));
  enqueue_c2r(h, h->ustage, h->pplain);
  HOS_CK(cudaGetLastError());
  HOS_CK(host_copy(u_phys, h->pplain, h->psz * sizeof(double), h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_check_finite(hos_handle h, int* finite) {
  if (!h || !finite) return fail(HOS_ERR_ARG, "null argument");
  HOS_CK(cudaMemsetAsync(h->flagdev, 0, sizeof(int), h->st));
  k_nonfinite<<<148, 256, 0, h->st>>>(h->u, 2 * h->fsz, h->flagdev);
  int f = 0;
  HOS_CK(cudaGetLastError());
  HOS_CK(cudaMemcpyAsync(&f, h->flagdev, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  *finite = f ? 0 : 1;
  return HOS_OK;
}

int hos_profile_stage(hos_handle h, double dt, int reps, hos_pass_stat* out, int max, int* count) {
  if (!h || !out || !count || reps < 1) return fail(HOS_ERR_ARG, "bad argument");
  // stage 1 of an RK step from the resident state, written to scratch: the
  // state, t and the energy record are untouched
  HOS_CK(cudaMemcpyAsync(h->ustage, h->u, 2 * h->fsz * sizeof(double2), cudaMemcpyDeviceToDevice, h->st));
  HOS_CK(cudaMemcpyAsync(h->trhs, h->tdev, sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  int act = 0;
  HOS_CK(cudaMemcpyAsync(&act, h->actdev, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  const int s = h->nst > 1 ? 1 : 0;
  double2* kout = h->k + (size_t)(h->nst - 1) * 2 * h->fsz;
  std::vector<double> ms(P_NKIND, 0.0), by(P_NKIND, 0.0);
  std::vector<int> n(P_NKIND, 0);
  for (int r = 0; r < reps; r++) {
    PassLog lg;
    lg.act_rows = act;
    log_pass(h, &lg, -1, 0.0);
    int rc = enqueue_stage(h, s, dt, true, h->ustage, kout, h->trhs, h->actdev, &lg);
    if (rc) return rc;
    HOS_CK(cudaStreamSynchronize(h->st));
    for (size_t i = 1; i < lg.ev.size(); i++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, lg.ev[i - 1], lg.ev[i]);
      const int k = lg.kind[i];
      ms[k] += t;
      by[k] += lg.bytes[i];
      if (r == 0) n[k]++;
    }
    for (cudaEvent_t e : lg.ev) cudaEventDestroy(e);
  }
  int c = 0;
  for (int k = 0; k < P_NKIND && c < max; k++) {
    if (!n[k]) continue;
    std::memset(&out[c], 0, sizeof(out[c]));
    std::strncpy(out[c].name, pass_name(k), sizeof(out[c].name) - 1);
    out[c].launches_per_stage = n[k];
    out[c].ms_per_launch = ms[k] / (reps * n[k]);
    out[c].bytes_per_launch = by[k] / (reps * n[k]);
    c++;
  }
  *count = c;
  HOS_CK(cudaGetLastError());
  return HOS_OK;
}

int hos_zvel(hos_handle h, const double* u, double* wM, double* wM2, double* w2M, double* w2M2) {
  if (!h || !u || !wM || !wM2 || !w2M || !w2M2) return fail(HOS_ERR_ARG, "null argument");
  if (!h->zvbuf) {
    int rc = dalloc_on(&h->zvbuf, 4 * h->fsz * sizeof(double2), h->st);
    if (rc) return rc;
  }
  HOS_CK(host_copy(h->ustage, u, 2 * h->fsz * sizeof(double2), h->st));
  int rc = enqueue_stage(h, 0, 0.0, true, h->ustage, nullptr, h->trhs, nullptr, nullptr, h->zvbuf);
  if (rc) return rc;
  HOS_CK(cudaGetLastError());
  double* outs[4] = {wM, wM2, w2M, w2M2};
  for (int q = 0; q < 4; q++)
    HOS_CK(host_copy(outs[q], h->zvbuf + (size_t)q * h->fsz, h->fsz * sizeof(double2), h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_spectral_op(hos_handle h, int op, const double* a, const double* b, double* out) {
  if (!h || !a || !out || ((op == HOS_OP_SUM || op == HOS_OP_MULT) && !b)) return fail(HOS_ERR_ARG, "null argument");
  if (op < HOS_OP_DX || op > HOS_OP_MULT) return fail(HOS_ERR_ARG, "unknown operator %d", op);
  if (!h->zvbuf) {
    int rc = dalloc_on(&h->zvbuf, 4 * h->fsz * sizeof(double2), h->st);
    if (rc) return rc;
  }
  double2* da = h->zvbuf;
  double2* db = h->zvbuf + h->fsz;
  double2* dout = h->zvbuf + 2 * h->fsz;
  HOS_CK(host_copy(da, a, h->fsz * sizeof(double2), h->st));
  if (b) HOS_CK(host_copy(db, b, h->fsz * sizeof(double2), h->st));
  if (op == HOS_OP_MULT) {  // Mult, operators_par.c:210-235
    enqueue_c2r(h, da, h->pplain);
    enqueue_c2r(h, db, h->pplain + h->psz);
    k_mul_real<<<296, 256, 0, h->st>>>(h->pplain, h->pplain + h->psz, h->pplain, h->psz);
    enqueue_r2c(h, h->pplain, dout, 0);
  } else {
    k_spec_op<<<296, 256, 0, h->st>>>(h->geo, op, da, db, dout);
  }
  HOS_CK(cudaGetLastError());
  HOS_CK(host_copy(out, dout, h->fsz * sizeof(double2), h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  return HOS_OK;
}

int hos_hamiltonian(hos_handle h, const double* eta, const double* eta_t, const double* phi, double* H) {
  if (!h || !eta || !eta_t || !phi || !H) return fail(HOS_ERR_ARG, "null argument");
  if (!h->zvbuf) {
    int rc = dalloc_on(&h->zvbuf, 4 * h->fsz * sizeof(double2), h->st);
    if (rc) return rc;
  }
  if (!h->hpart) {
    int rc = dalloc_on(&h->hpart, (size_t)(h->h + 2) * sizeof(double), h->st);
    if (rc) return rc;
  }
  const double* src[3] = {eta, eta_t, phi};
  for (int q = 0; q < 3; q++)
    HOS_CK(host_copy(h->zvbuf + (size_t)q * h->fsz, src[q], h->fsz * sizeof(double2), h->st));
  k_ham_rows<<<h->h + 1, 256, 0, h->st>>>(h->geo, h->zvbuf, h->zvbuf + h->fsz, h->zvbuf + 2 * h->fsz, h->hpart);
  k_sum_parts<<<1, 256, 0, h->st>>>(h->hpart, h->h + 1, h->hpart + h->h + 1);
  HOS_CK(cudaGetLastError());
  double r = 0.0;
  HOS_CK(cudaMemcpyAsync(&r, h->hpart + h->h + 1, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  *H = r;
  return HOS_OK;
}

int hos_ensemble_create(const hos_handle* members, const double* dt, int n, hos_ensemble* out) {
  return hos_ensemble_create_ex(members, dt, n, HOS_ENS_CLASSES, out);
}

int hos_ensemble_create_ex(const hos_handle* members, const double* dt, int n, int mode, hos_ensemble* out) {
  if (!members || !dt || !out || n < 1) return fail(HOS_ERR_ARG, "bad argument");
  if (mode != HOS_ENS_CLASSES && mode != HOS_ENS_PERSISTENT) return fail(HOS_ERR_ARG, "unknown ensemble mode %d", mode);
  *out = nullptr;
  hos_ens* E = new hos_ens();
  E->mode = mode;
  for (int i = 0; i < n; i++) {
    if (!members[i]) {
      delete E;
      return fail(HOS_ERR_ARG, "null member %d", i);
    }
    for (int j = 0; j < i; j++)
      if (members[j] == members[i]) {
        delete E;
        return fail(HOS_ERR_ARG, "member %d appears twice", i);
      }
    E->mem.push_back(members[i]);
    E->dt.push_back(dt[i]);
  }
  for (int i = 0; i < n; i++) {
    size_t ci = 0;
    for (; ci < E->cls.size(); ci++)
      if (same_class(E->mem[E->cls[ci].idx[0]], E->mem[i])) break;
    if (ci == E->cls.size()) E->cls.emplace_back();
    if (E->cls[ci].idx.size() >= 65535) {
      release_ens(E);
      return fail(HOS_ERR_ARG, "more than 65535 members of one size class");
    }
    E->cls[ci].idx.push_back(i);
  }
  cudaError_t err = cudaStreamCreateWithFlags(&E->st, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&E->fork, cudaEventDisableTiming);
  for (EnsClass& K : E->cls) {
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&K.st, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&K.join, cudaEventDisableTiming);
  }
  if (err != cudaSuccess) {
    release_ens(E);
    return fail(HOS_ERR_CUDA, "ensemble streams: %s", cudaGetErrorString(err));
  }
  // members' pending work (state uploads) completes before the first step
  for (hos_ctx* c : E->mem) {
    err = cudaStreamSynchronize(c->st);
    if (err != cudaSuccess) {
      release_ens(E);
      return fail(HOS_ERR_CUDA, "member sync: %s", cudaGetErrorString(err));
    }
  }
  int rc = dalloc(&E->any_bad, sizeof(int));
  if (rc == HOS_OK && cudaMemset(E->any_bad, 0, sizeof(int)) != cudaSuccess) rc = fail(HOS_ERR_CUDA, "memset");
  if (rc == HOS_OK) rc = dalloc(&E->rem_cls, (size_t)n * sizeof(int));
  if (rc == HOS_OK && cudaMemset(E->rem_cls, 0xff, (size_t)n * sizeof(int)) != cudaSuccess)
    rc = fail(HOS_ERR_CUDA, "memset");  // -1: no budget
  if (rc) {
    release_ens(E);
    return rc;
  }
  if (E->mode == HOS_ENS_PERSISTENT) {
    for (size_t i = 1; i < E->mem.size(); i++)
      if (E->mem[i]->device != E->mem[0]->device) {
        release_ens(E);
        return fail(HOS_ERR_ARG, "persistent ensemble: members on different devices");
      }
    int dev0 = 0;
    cudaGetDevice(&dev0);
    cudaSetDevice(E->mem[0]->device);
    rc = plan_persist(E);
    cudaSetDevice(dev0);
  } else {
    rc = build_ens_graph(E);
  }
  if (rc) {
    release_ens(E);
    return rc;
  }
  *out = E;
  return HOS_OK;
}

int hos_ensemble_step(hos_ensemble e, int nsteps) {
  if (!e || nsteps < 0) return fail(HOS_ERR_ARG, "bad argument");
  if (e->mode == HOS_ENS_PERSISTENT) {
    for (int i = 0; i < nsteps; i++) HOS_CK(persist_launch(e->pa, e->pblocks, e->psmem, e->st, e->minb));
    return HOS_OK;
  }
  for (int i = 0; i < nsteps; i++) HOS_CK(cudaGraphLaunch(e->gexec, e->st));
  return HOS_OK;
}

int hos_ensemble_set_wait_limit(hos_ensemble e, long long ns) {
  if (!e || ns <= 0) return fail(HOS_ERR_ARG, "bad argument");
  e->pa.wait_limit_ns = ns;
  return HOS_OK;
}

int hos_ensemble_set_steps(hos_ensemble e, const int* steps) {
  if (!e || !steps) return fail(HOS_ERR_ARG, "null argument");
  int* rem = e->mode == HOS_ENS_PERSISTENT ? e->pa.remaining : e->rem_cls;
  HOS_CK(cudaMemcpyAsync(rem, steps, e->mem.size() * sizeof(int), cudaMemcpyHostToDevice, e->st));
  HOS_CK(cudaStreamSynchronize(e->st));
  return HOS_OK;
}

int hos_ensemble_get_remaining(hos_ensemble e, int* steps) {
  if (!e || !steps) return fail(HOS_ERR_ARG, "null argument");
  const int* rem = e->mode == HOS_ENS_PERSISTENT ? e->pa.remaining : e->rem_cls;
  HOS_CK(cudaMemcpyAsync(steps, rem, e->mem.size() * sizeof(int), cudaMemcpyDeviceToHost, e->st));
  HOS_CK(cudaStreamSynchronize(e->st));
  return HOS_OK;
}

int hos_ensemble_withhold_dependency(hos_ensemble e, int on) {
  if (!e) return fail(HOS_ERR_ARG, "null ensemble");
  if (e->mode != HOS_ENS_PERSISTENT) return fail(HOS_ERR_STATE, "only persistent ensembles have work lists");
  HOS_CK(cudaStreamSynchronize(e->st));
  e->withhold = on ? 1 : 0;
  return plan_persist(e);
}

int hos_ensemble_sync(hos_ensemble e) {
  if (!e) return fail(HOS_ERR_ARG, "null ensemble");
  HOS_CK(cudaStreamSynchronize(e->st));
  HOS_CK(cudaGetLastError());
  if (e->mode == HOS_ENS_PERSISTENT) {
    int err = 0;
    HOS_CK(cudaMemcpy(&err, e->pa.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
      long long info[4] = {0, 0, 0, 0};
      HOS_CK(cudaMemcpy(info, e->pa.err_info, sizeof(info), cudaMemcpyDeviceToHost));
      HOS_CK(cudaMemset(e->pa.err, 0, sizeof(int)));
      return fail(HOS_ERR_TIMEOUT,
                  "persistent ensemble: item %lld of member %lld waited past the limit for %lld completed items "
                  "(saw %lld); the members' states are not valid until set again",
                  info[0], info[1], info[2], info[3]);
    }
  }
  int bad = 0;
  HOS_CK(cudaMemcpy(&bad, e->any_bad, sizeof(int), cudaMemcpyDeviceToHost));
  if (bad) return fail(HOS_ERR_NONFINITE, "a member's state became non-finite (hos_health on each member tells which)");
  return HOS_OK;
}

void* hos_ensemble_stream(hos_ensemble e) { return e ? (void*)e->st : nullptr; }

int hos_ensemble_info(hos_ensemble e, int* nclasses, int* launches_per_step) {
  if (!e) return fail(HOS_ERR_ARG, "null ensemble");
  if (nclasses) *nclasses = e->mode == HOS_ENS_PERSISTENT ? 1 : (int)e->cls.size();
  if (launches_per_step) *launches_per_step = e->launches_per_step;
  return HOS_OK;
}

int hos_ensemble_destroy(hos_ensemble e) {
  if (!e) return HOS_OK;
  cudaStreamSynchronize(e->st);
  release_ens(e);
  return HOS_OK;
}

int hos_launches_per_step(hos_handle h) {
  if (!h) return -1;
  const int per_stage = 4 + 3 * h->L - (h->cfg.ec.fuse && h->L >= 2 ? h->L - 1 : 0);
  return h->nst * per_stage + 1;
}

int hos_volume(hos_handle h, double* vol) {
  if (!h || !vol) return fail(HOS_ERR_ARG, "null argument");
  double2 v;
  HOS_CK(cudaMemcpyAsync(&v, h->u, sizeof(double2), cudaMemcpyDeviceToHost, h->st));
  HOS_CK(cudaStreamSynchronize(h->st));
  *vol = v.x;
  return HOS_OK;
}

}  // extern "C"
