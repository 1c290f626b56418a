// hos_fft_2d_noalloc: the normalised 2-D real-to-complex transform of fft_2d
// without any memory allocation, for callers that cannot allocate GPU
// memory themselves or let a library do it:
//   * code that runs while a CUDA stream is being captured into a graph,
//     where cudaMalloc / cudaFree are not permitted;
//   * latency-critical loops, where cudaMalloc / cudaFree would synchronise
//     the whole device;
//   * host programs that give all device memory to their own allocator and
//     forbid allocations from outside it.
// The caller passes the physical input and the spectral output (device
// memory) and a stream.  The intermediate half spectrum lives in a
// file-scope device array of fixed size, and the twiddle tables in another,
// filled on the device at every call; neither is ever allocated or freed.
//
// Limits: nx and ny powers of two in [16, 2048] and nx*(ny/2+1) <= 525312
// complex values (for example 1024 x 1024); larger grids are rejected with
// HOS_ERR_ARG.  Every GPU that loads the library holds the arrays (about
// 8.5 MB) until the process exits.
//
// The arrays are shared by every call on a device: calls that overlap on the
// GPU (for example on two streams without an order between them) race and
// must not be issued.  The scratch needs no clearing: the first pass writes
// every element the second pass reads.
#include <cstdio>
#include <mutex>
#include <string>

#include "hos_gpu.h"
#include "hos_registry.h"

namespace hos {
void set_last_error(const char* msg);
}

namespace {

constexpr size_t NOALLOC_MAX_SPEC = 1024 * 513;  // complex values of the intermediate
constexpr int NOALLOC_MAX_LEN = 2048;            // longest line (nx, ny)
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double2 g_noalloc_spec[NOALLOC_MAX_SPEC];
static __device__ __align__(256) double2 g_noalloc_tw[3 * NOALLOC_MAX_LEN];

struct DevPtrs {
  double2* spec = nullptr;
  double2* tw = nullptr;
  unsigned long long ctx_id = 0;  // the context the addresses belong to
  bool ready = false;
};
DevPtrs g_dev[NOALLOC_MAX_DEVICES];
std::mutex g_mu;

// exp(-2 pi i k / n) for the three line lengths of a call, in the layout
// [nx | ny/2 | ny] at stride NOALLOC_MAX_LEN.
__global__ void k_noalloc_twiddles(double2* tw, int nx, int h, int ny) {
  const int lens[3] = {nx, h, ny};
  for (int q = 0; q < 3; q++) {
    const int n = lens[q];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
      double s, c;
      sincospi(2.0 * (double)k / (double)n, &s, &c);
      tw[q * NOALLOC_MAX_LEN + k] = make_double2(c, -s);
    }
  }
}

int fail(int code, const char* msg) {
  hos::set_last_error(msg);  // reported by hos_last_error()
  return code;
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Unique id of the calling thread's current context (driver entry points
// cuCtxGetCurrent / cuCtxGetId, fetched through the runtime so that the
// library needs no link against the driver library); 0 if unavailable.
unsigned long long current_context_id() {
  typedef int (*GetCurrentFn)(void**);
  typedef int (*GetIdFn)(void*, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(f);
    (void)cudaGetLastError();
  });
  void* c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != 0 || !c || get_id(c, &id) != 0) return 0;
  return id;
}

// Set-up per device: the device addresses of the two arrays, taken with the
// device current.  It runs on the first call on a device, and again if that
// device's context has since been replaced (cudaDeviceReset, which reloads
// the library's device code at new addresses).
int setup_device(int dev, DevPtrs** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(HOS_ERR_ARG, "device index out of range");
  const unsigned long long cid = current_context_id();  // 0: no context current on this thread yet
  std::lock_guard<std::mutex> lk(g_mu);
  DevPtrs& d = g_dev[dev];
  if (d.ready && cid != d.ctx_id) d.ready = false;
  if (!d.ready) {
    cudaError_t e = cudaGetSymbolAddress((void**)&d.spec, g_noalloc_spec);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.tw, g_noalloc_tw);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return fail(HOS_ERR_CUDA, cudaGetErrorString(e));
    }
    d.ctx_id = current_context_id();  // the lookup made the device's context current
    d.ready = true;
  }
  *out = &d;
  return HOS_OK;
}

}  // namespace

extern "C" int hos_fft_2d_noalloc(const double* u_phys, double* hu, int nx, int ny, void* stream) {
  using namespace hos;
  if (!u_phys || !hu) return fail(HOS_ERR_ARG, "null pointer");
  if (!pow2(nx) || !pow2(ny) || nx < 16 || ny < 16 || nx > NOALLOC_MAX_LEN || ny > NOALLOC_MAX_LEN)
    return fail(HOS_ERR_ARG, "nx, ny must be powers of two in [16, 2048]");
  const int h = ny / 2;
  if ((size_t)nx * (size_t)(h + 1) > NOALLOC_MAX_SPEC)
    return fail(HOS_ERR_ARG, "grid too large: nx*(ny/2+1) must not exceed 525312");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return fail(HOS_ERR_CUDA, "cudaGetDevice failed");
  }
  DevPtrs* d = nullptr;
  int rc = setup_device(dev, &d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;

  // the double-precision pass kernels of fft_2d with 8 elements per thread
  const int ex = 8, ey = 8;
  YFwdFn yf = lookup_yfwd(0, YF_PLAIN, h, ey);
  XFwdFn xf = lookup_xfwd(0, XF_PLAIN, nx, ex);
  if (!yf || !xf) return fail(HOS_ERR_ARG, "no kernels for this grid");
  const int py = h / ey;
  int gy = MAX_THREADS / py;
  if (gy > nx) gy = nx;
  if (gy < 1) gy = 1;
  int lp = h + 1;
  while (lp % 8 != (gy >= 8 ? 1 : 8 / gy) % 8) lp++;
  const int px = nx / ex;
  int gx = 128 / px;
  if (gx < 1) gx = 1;

  Geo geo{};
  geo.nx = nx;
  geo.ny = ny;
  geo.h = h;
  geo.mx = nx;  // no dealiasing on this path
  geo.my = h + 1;
  geo.inv_nxny = 1.0 / ((double)nx * (double)ny);

  k_noalloc_twiddles<<<8, 256, 0, st>>>(d->tw, nx, h, ny);

  YFwdArgs fa{};
  fa.geo = geo;
  fa.lp = lp;
  fa.in_ptr = u_phys;
  fa.vout = d->spec;
  fa.rows_out = h + 1;
  yf<<<dim3(nx / gy, 1), gy * py, (size_t)gy * lp * sizeof(double2), st>>>(fa, nullptr, d->tw + NOALLOC_MAX_LEN,
                                                                            d->tw + 2 * NOALLOC_MAX_LEN);
  XFwdArgs xa{};
  xa.geo = geo;
  xa.rows = h + 1;
  xa.vin0 = d->spec;
  xa.out_spec = reinterpret_cast<double2*>(hu);
  xa.dealias = 0;
  xf<<<dim3((h + 1 + gx - 1) / gx, 1), gx * px, (size_t)gx * nx * sizeof(double2), st>>>(xa, nullptr, d->tw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(HOS_ERR_CUDA, cudaGetErrorString(e));
  return HOS_OK;
}
