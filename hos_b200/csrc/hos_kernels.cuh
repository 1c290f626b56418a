// Pass kernels of the HOS right-hand side on sm_100a.
//
// Spectral fields use the reference's single-rank TRANSPOSED_OUT layout:
// complex [Ny/2+1][Nx], ky-major, kx contiguous (fft_routines_2d_par.c:37 via
// main_2d_par.c:189).  Physical fields are unpadded real [Nx][Ny].  Every 2-D
// transform is two passes:
//
//   c2r: x-pass (inverse complex DFT along kx of each ky row, contiguous)
//        -> Z [Ny/2+1][Nx] -> y-pass (complex-to-real along y of each x row)
//   r2c: y-pass (real-to-complex along y of each x row) -> V [Ny/2+1][Nx]
//        -> x-pass (complex DFT along x of each ky row)
//
// x-passes read and write whole rows with consecutive threads on consecutive
// addresses.  y-passes own G consecutive x rows; their spectral side is read
// or written as G-wide column strips staged through shared memory, in the
// same buffer the line FFT then uses for its exchanges.
//
// Kernels are specialised per mode (so each mode gets its own register
// allocation) and most take one output per block along gridDim.y, which
// keeps many small blocks resident per SM; inputs that several outputs share
// are re-read from L2.
//
// The spectral multipliers, the RK stage input, the Taylor products of the
// vertical-velocity recursion, the RHS assembly, the Dommermuth ramp, the
// dealias mask, the stage-0 Hamiltonian and the final RK update are fused
// into the prologues and epilogues of these passes.
#pragma once

#include "fft_line.cuh"

namespace hos {

constexpr int MAX_STAGES = 7;
constexpr int MAX_JOBS = 16;
constexpr int MAX_TERMS = 8;
constexpr int MAX_THREADS = 256;

struct Geo {
  int nx, ny, h;   // h = ny/2
  int mx, my;      // dealias bounds (operators_par.c:290-291)
  double kx0, ky0; // 2 pi / Lx, 2 pi / Ly
  double depth;    // <= 0: deep water
  double g;
  double inv_nxny;
};

// kx of spectral column i, with the reference's convention that
// i <= Nx/2 + 1 is positive (operators_par.c:55-63, :173).
__device__ __forceinline__ double kx_of(const Geo& G, int i) {
  return (i <= G.nx / 2 + 1) ? (double)i * G.kx0 : -(double)(G.nx - i) * G.kx0;
}
__device__ __forceinline__ double ky_of(const Geo& G, int j) { return (double)j * G.ky0; }
__device__ __forceinline__ bool keep_mode(const Geo& G, int i, int j) {
  return !((i >= G.mx && i < G.nx - G.mx + 1) || j >= G.my);  // operators_par.c:314
}
// Multiplier of the p-th z-derivative: kz^p (deep water, operators_par.c:168-192);
// finite depth: kz^p * tanh(kz h) for odd p.
__device__ __forceinline__ double dz_mult(const Geo& G, double kz, int p) {
  double m = 1.0;
  for (int q = 0; q < p; q++) m *= kz;
  if ((p & 1) && G.depth > 0) m *= tanh(kz * G.depth);
  return m;
}

// The same multiplier at the compute precision T of a pass: in single
// precision it only scales single-precision data, so it is formed in single
// precision too (kx, ky and the quirky kx convention as in kx_of).
template <typename T>
__device__ __forceinline__ T dz_mult_t(const Geo& G, int i, int j, int p);
template <>
__device__ __forceinline__ double dz_mult_t<double>(const Geo& G, int i, int j, int p) {
  const double kx = kx_of(G, i), ky = ky_of(G, j);
  return dz_mult(G, sqrt(kx * kx + ky * ky), p);
}
// Wavenumbers in the compute precision T (single precision: formed from the
// integer mode index and the single-precision 2 pi / L, no double arithmetic).
template <typename T>
__device__ __forceinline__ T kx_t(const Geo& G, int i) {
  return (T)kx_of(G, i);
}
template <>
__device__ __forceinline__ float kx_t<float>(const Geo& G, int i) {
  return (float)(i <= G.nx / 2 + 1 ? i : i - G.nx) * (float)G.kx0;
}
template <typename T>
__device__ __forceinline__ T ky_t(const Geo& G, int j) {
  return (T)ky_of(G, j);
}
template <>
__device__ __forceinline__ float ky_t<float>(const Geo& G, int j) {
  return (float)j * (float)G.ky0;
}
template <>
__device__ __forceinline__ float dz_mult_t<float>(const Geo& G, int i, int j, int p) {
  const float kx = kx_t<float>(G, i), ky = ky_t<float>(G, j);
  const float kz = sqrtf(kx * kx + ky * ky);
  float m = 1.0f;
  for (int q = 0; q < p; q++) m *= kz;
  if ((p & 1) && G.depth > 0) m *= tanhf(kz * (float)G.depth);
  return m;
}

// Programmatic dependent launch.  The engine launches the passes of a step
// with programmatic stream serialisation, so a pass can be launched and its
// blocks placed while the previous pass drains.  Every such kernel first
// waits for the previous grid to complete and its writes to be visible
// (before it reads or writes global memory), then allows the next pass to
// launch.  Launched without the attribute both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

enum { XI_STAGE = 0, XI_PLAIN = 1 };
enum { XF_PLAIN = 0, XF_LEVEL = 1, XF_RHS = 2 };
enum { YI_JOBS = 0, YI_LEVEL = 1 };
enum { YF_PLAIN = 0, YF_LEVEL = 1, YF_RHS = 2 };

// ---------------------------------------------------------------- x inverse
struct XInvArgs {
  Geo geo;
  const int* remaining; // batched launches: the member's step budget (0: skip the pass); nullptr: no budget
  int ycount;           // batched launches: blocks with blockIdx.y >= ycount have no work
  int rows;             // ky rows that may be nonzero in the input
  const int* rows_dev;  // if set, overrides rows (active rows of the state, kept on the device)
  const double2* u;     // STAGE: packed state [2][h+1][nx]; PLAIN: one field
  const double2* kp[MAX_STAGES];  // earlier stage derivatives
  double coef[MAX_STAGES];        // dt*b[s][p]
  int nk;
  void* z;              // output complex arrays (T2), stride (h+1)*nx; output o = blockIdx.y
  double2* ustg;        // STAGE: the stage input is also stored here ([2][h+1][nx], rows < rows)
  const double* tdev;   // simulation time (device)
  double* rdev;         // ramp factor for this step (device), written if set_ramp
  int set_ramp;
  double tramp;
  int rampflg;
};

// STAGE outputs (blockIdx.y = o): 0 eta, 1 i kx eta, 2 phi, 3 i kx phi,
// 3+p d_z^p phi (p >= 1).  The stage input u + sum coef*k is formed on the
// fly (time_schemes_par.c:38-67).
// Pass bodies.  Every pass is written as a device function of the block's
// coordinates (bx, by) and its thread count, so that the same code runs as a
// kernel of its own (the wrappers below pass blockIdx and blockDim) and as a
// work item of the persistent ensemble kernel (hos_persist.cu), which gives
// each item a virtual block.  smraw is the block's dynamic shared memory.
template <typename T, int NX, int E, int MODE>
__device__ __forceinline__ void xinv_body(const XInvArgs& a, int bx, int by, int nthreads, const void* twv,
                                          unsigned char* smraw) {
  using C = cpx<T>;
  constexpr int P = NX / E;
  const C* tw = reinterpret_cast<const C*>(twv);
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* sm = reinterpret_cast<C*>(smraw) + line * line_smem_elems<NX, E>();
  const int lines = nthreads / P;
  const int row = bx * lines + line;
  const int rows = a.rows_dev ? *a.rows_dev : a.rows;
  const Geo& geo = a.geo;
  const size_t fsz = (size_t)(geo.h + 1) * NX;
  const int o = by;

  if (MODE == XI_STAGE && a.set_ramp && bx == 0 && o == 0 && threadIdx.x == 0) {
    double r = 1.0;
    if (a.rampflg == 1) {
      const double tt = *a.tdev;
      r = 1 - exp(-tt * tt / a.tramp / a.tramp);  // RampFun, hosm_2d_par.c:526-530
    }
    *a.rdev = r;
  }
  if (bx * lines >= rows) return;  // whole block beyond the active rows
  const bool live = row < rows;
  const size_t roff = (size_t)(live ? row : 0) * NX;
  C* z = reinterpret_cast<C*>(a.z) + (size_t)o * fsz;

  C v[E];
  if (MODE == XI_PLAIN) {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = live ? conv<T>(a.u[roff + t + e * P]) : mkc((T)0, (T)0);
  } else {
    const size_t foff = (o < 2) ? 0 : fsz;
#pragma unroll
    for (int e = 0; e < E; e++) {
      double2 x = make_double2(0.0, 0.0);
      const int i = t + e * P;
      if (live) {
        const size_t idx = foff + roff + i;
        x = a.u[idx];
        for (int p = 0; p < a.nk; p++) {
          const double2 kk = a.kp[p][idx];
          x.x = x.x + a.coef[p] * kk.x;
          x.y = x.y + a.coef[p] * kk.y;
        }
      }
      if ((o == 0 || o == 2) && live) a.ustg[foff + roff + i] = x;
      if (o == 1 || o == 3) {  // Dx: i kx (operators_par.c:66)
        const T kx = kx_t<T>(geo, i);
        const C xc = conv<T>(x);
        v[e] = mkc(-kx * xc.y, kx * xc.x);
      } else if (o >= 4) {  // Dz applied o-3 times (operators_par.c:168-192)
        v[e] = cscale(conv<T>(x), dz_mult_t<T>(geo, i, row, o - 3));
      } else {
        v[e] = conv<T>(x);
      }
    }
  }
  line_fft<T, NX, E, true>(v, sm, t, tw);
  if (live) {
#pragma unroll
    for (int e = 0; e < E; e++) z[roff + t + e * P] = v[e];
  }
}

template <typename T, int NX, int E, int MODE, bool B>
__global__ void __launch_bounds__(MAX_THREADS, 2) k_xinv(const __grid_constant__ XInvArgs a0,
                                                         const XInvArgs* __restrict__ arr, const void* twv) {
  pdl_enter();
  const XInvArgs& a = B ? arr[blockIdx.z] : a0;  // batched: one field per z
  if (B && (int)blockIdx.y >= a.ycount) return;
  if (B && a.remaining && *a.remaining == 0) return;  // the member's step budget is spent
  extern __shared__ __align__(16) unsigned char smraw[];
  xinv_body<T, NX, E, MODE>(a, blockIdx.x, blockIdx.y, blockDim.x, twv, smraw);
}

// ---------------------------------------------------------------- x forward
struct XFwdArgs {
  Geo geo;
  const int* remaining; // batched launches: the member's step budget (0: skip the pass); nullptr: no budget
  int ycount;           // batched launches: blocks with blockIdx.y >= ycount have no work
  int rows;             // rows processed
  const int* rows_dev;  // if set, overrides rows
  int rows_fft;         // RHS: rows < rows_fft are transformed; rows in [rows_fft, rows) only add to the Hamiltonian
  const void* vin0;     // input V arrays (T2) [h+1][nx]; RHS: blockIdx.y selects vin0 (eta) or vin1 (phi)
  const void* vin1;
  double2* out_spec;    // PLAIN output; blockIdx.y = q reads vin0 + q*fsz and writes out_spec + q*fsz
  int dealias;          // PLAIN: zero the modes Dealias zeroes (operators_par.c:283-325)
  int addk_mask;        // PLAIN: bit q set -> add Dz of the phi field of u_add to output q (W^(1), hosm_2d_par.c:280-288)
  const double2* u_add; // PLAIN: packed state whose phi field supplies that term
  void* zout;           // LEVEL: output Z arrays (T2), stride (h+1)*nx
  int ndz;              // LEVEL: z-derivative orders 1..ndz
  int opb;              // LEVEL: orders per block (blockIdx.y covers orders y*opb+1 ..)
  // RHS
  double2* u;                     // packed state at step start (updated in place on the final stage)
  const double2* ustg;            // stage input of both fields, written by the x-inverse pass
                                  // (never read from u: on the final stage the other field's
                                  // blocks overwrite u)
  double2* kout;                  // this stage's derivative [2][h+1][nx]
  const double* rdev;             // ramp factor
  int ham;                        // accumulate the stage-0 Hamiltonian
  double* ham_part;               // one partial per ky row (h+1 of them)
  int final_update;               // u += sum cfin[s] * k_s (time_schemes_par.c:98-116)
  const double2* kall[MAX_STAGES];
  double cfin[MAX_STAGES];
  int nstage;                     // number of stages; k of the last one is in registers
};

template <typename T, int NX, int E, int MODE>
__device__ __forceinline__ void xfwd_body(const XFwdArgs& a, int bx, int by, int nthreads, const void* twv,
                                          unsigned char* smraw) {
  using C = cpx<T>;
  constexpr int P = NX / E;
  const C* tw = reinterpret_cast<const C*>(twv);
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* sm = reinterpret_cast<C*>(smraw) + line * line_smem_elems<NX, E>();
  const int lines = nthreads / P;
  const int row = bx * lines + line;
  const Geo& geo = a.geo;
  const size_t fsz = (size_t)(geo.h + 1) * NX;

  if (MODE != XF_RHS) {
    const T sc = (T)geo.inv_nxny;
    const bool live = row < a.rows;
    const size_t roff = (size_t)(live ? row : 0) * NX;
    const C* vin = reinterpret_cast<const C*>(a.vin0) + (MODE == XF_PLAIN ? (size_t)by * fsz : 0);
    C v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = live ? vin[roff + t + e * P] : mkc((T)0, (T)0);
    line_fft<T, NX, E, false>(v, sm, t, tw);
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = cscale(v[e], sc);  // fft_2d's 1/Nx/Ny (exact: powers of two)
    if (MODE == XF_PLAIN) {
      if (live) {
        double2* out = a.out_spec + (size_t)by * fsz;
        const bool addk = (a.addk_mask >> by) & 1;
        const double ky = ky_of(geo, row);
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int i = t + e * P;
          const bool z0 = a.dealias && !keep_mode(geo, i, row);
          double2 r = z0 ? make_double2(0.0, 0.0) : widen(v[e]);
          if (addk) {
            const double kx = kx_of(geo, i);
            const double m1 = dz_mult(geo, sqrt(kx * kx + ky * ky), 1);
            const double2 ph = a.u_add[fsz + roff + i];
            r.x += m1 * ph.x;
            r.y += m1 * ph.y;
          }
          out[roff + i] = r;
        }
      }
      return;
    }
    // LEVEL: v holds phi^(n+1) hat; this block emits its z-derivatives of
    // orders p0+1 .. p0+opb, p0 = by*opb (the forward transform is
    // repeated per block, so opb trades repeated work for parallel blocks)
    const int p0 = by * a.opb;
    const int p1 = min(p0 + a.opb, a.ndz);
    for (int p = p0 + 1; p <= p1; p++) {
      C w[E];
#pragma unroll
      for (int e = 0; e < E; e++) w[e] = cscale(v[e], dz_mult_t<T>(geo, t + e * P, row, p));
      line_fft<T, NX, E, true>(w, sm, t, tw);
      if (live) {
        C* z = reinterpret_cast<C*>(a.zout) + (size_t)(p - 1) * fsz;
#pragma unroll
        for (int e = 0; e < E; e++) z[roff + t + e * P] = w[e];
      }
    }
    return;
  }

  // ---- RHS: end of an RK stage (rhs_hos tail, hosm_2d_par.c:181-233, and
  // sol_update_RK bookkeeping, time_schemes_par.c:70-116).  by = 0
  // finishes eta_t (and the Hamiltonian), by = 1 finishes phi_t.
  __shared__ double red[MAX_THREADS / 32];
  const int f = by;
  const int rows = a.rows_dev ? *a.rows_dev : a.rows;
  const bool live = row < rows;
  const bool fft_row = row < a.rows_fft;
  const size_t roff = (size_t)(live ? row : 0) * NX;
  const bool block_fft = bx * lines < a.rows_fft;
  C v[E];
  if (block_fft) {
    const C* vin = reinterpret_cast<const C*>(f == 0 ? a.vin0 : a.vin1);
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = fft_row ? vin[roff + t + e * P] : mkc((T)0, (T)0);
    line_fft<T, NX, E, false>(v, sm, t, tw);
  } else {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = mkc((T)0, (T)0);
  }
  double hacc = 0.0;
  if (live && (fft_row || (f == 0 && a.ham))) {
    const double ky = ky_of(geo, row);
    const double R = *a.rdev;
    const double wrow = (row == 0) ? 1.0 : 2.0;  // Hamiltonian weights, hosm_2d_par.c:473-519
    const size_t mine = f == 0 ? 0 : fsz, other = f == 0 ? fsz : 0;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int i = t + e * P;
      const size_t idx = roff + i;
      const double2 u0 = a.u[mine + idx];   // this field at step start
      const double2 uo = a.ustg[other + idx];  // the other field's stage input (= u at stage 0)
      double2 kt = make_double2(0.0, 0.0);
      if (fft_row && keep_mode(geo, i, row)) {
        const double2 s = cscale(widen(v[e]), geo.inv_nxny);
        if (f == 0) {  // eta_t = R * NL_eta + Dz phi
          const double kx = kx_of(geo, i);
          const double m1 = dz_mult(geo, sqrt(kx * kx + ky * ky), 1);
          kt.x = R * s.x + m1 * uo.x;
          kt.y = R * s.y + m1 * uo.y;
        } else {  // phi_t = R * NL_phi - g eta
          kt.x = R * s.x - geo.g * uo.x;
          kt.y = R * s.y - geo.g * uo.y;
        }
      }
      if (fft_row) a.kout[mine + idx] = kt;
      if (f == 0 && a.ham)  // g|eta|^2 + Re(phi conj(eta_t)) at step start (stage 0: stage input = u)
        hacc += wrow * (geo.g * u0.x * u0.x + geo.g * u0.y * u0.y + uo.x * kt.x + uo.y * kt.y);
      if (a.final_update && fft_row) {
        double2 nu = u0;
        for (int s = 0; s + 1 < a.nstage; s++) {
          const double2 k0 = a.kall[s][mine + idx];
          nu.x = nu.x + a.cfin[s] * k0.x;
          nu.y = nu.y + a.cfin[s] * k0.y;
        }
        const double cl = a.cfin[a.nstage - 1];
        nu.x = nu.x + cl * kt.x;
        nu.y = nu.y + cl * kt.y;
        a.u[mine + idx] = nu;
      }
    }
  }
  if (f == 0 && a.ham) {
    // one partial per ky row, summed over the row's P threads by a fixed
    // tree, so that the partials (and the energy the step end forms from
    // them) do not depend on how many rows a block holds
    if (P <= 32) {
      for (int off = P / 2; off > 0; off >>= 1) hacc += __shfl_down_sync(0xffffffffu, hacc, off, P);
      if (t == 0 && row <= geo.h) a.ham_part[row] = hacc;
    } else {
      for (int off = 16; off > 0; off >>= 1) hacc += __shfl_down_sync(0xffffffffu, hacc, off);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = hacc;
      __syncthreads();
      if (t == 0 && row <= geo.h) {
        double s = 0.0;
        for (int wi = 0; wi < P / 32; wi++) s += red[(threadIdx.x >> 5) + wi];
        a.ham_part[row] = s;
      }
    }
  }
}

template <typename T, int NX, int E, int MODE, bool B>
__global__ void __launch_bounds__(MAX_THREADS, 2) k_xfwd(const __grid_constant__ XFwdArgs a0,
                                                         const XFwdArgs* __restrict__ arr, const void* twv) {
  pdl_enter();
  const XFwdArgs& a = B ? arr[blockIdx.z] : a0;
  if (B && (int)blockIdx.y >= a.ycount) return;
  if (B && a.remaining && *a.remaining == 0) return;  // the member's step budget is spent
  extern __shared__ __align__(16) unsigned char smraw[];
  xfwd_body<T, NX, E, MODE>(a, blockIdx.x, blockIdx.y, blockDim.x, twv, smraw);
}

// Forward y-transform of the values v (pairs of physical points of this
// thread's line), real-to-complex postprocessing, and the transposed store of
// rows ky < rows_out of the G lines into the [h+1][nx] array vo.  All threads
// of the block must call it.
template <typename T, int H, int E>
__device__ __forceinline__ void yfwd_finish(cpx<T> (&v)[E], cpx<T>* sm, cpx<T>* tl, int t, int G, int lp,
                                            const cpx<T>* tw, const cpx<T>* twy, cpx<T>* vo, int nx, int ix0,
                                            int rows_out, int nthreads) {
  using C = cpx<T>;
  constexpr int P = H / E;
  line_fft<T, H, E, false>(v, tl, t, tw);
  // C[k] natural order -> line region, then real-to-complex postprocessing in
  // place, one (k, H-k) pair per thread slot
  __syncthreads();
#pragma unroll
  for (int e = 0; e < E; e++) tl[(t + e * P)] = v[e];
  __syncthreads();
#pragma unroll
  for (int e = 0; e <= E / 2; e++) {
    int k;
    if (e < E / 2) k = t + e * P;  // pairs (k, H-k), k in [0, H/2)
    else if (t == 0) k = H / 2;    // the self-paired middle bin
    else break;
    const int kn = H - k;  // partner; for k = 0 the partner is the Nyquist bin H (C[H] = C[0])
    const C ck = tl[(k)];
    const C cq = tl[(kn & (H - 1))];
    // X[k] = (C[k] + conj C[H-k])/2 + w^k (C[k] - conj C[H-k])/(2i),  w = exp(-2 pi i / Ny)
    const C cn = cconj(cq);
    const C ev = cscale(cadd(ck, cn), (T)0.5);
    const C d = csub(ck, cn);
    const C od = mkc((T)0.5 * d.y, (T)-0.5 * d.x);
    const C xk = cadd(ev, cmul(__ldg(&twy[k]), od));
    if (k != kn) {
      const C cm = cconj(ck);
      const C ev2 = cscale(cadd(cq, cm), (T)0.5);
      const C d2 = csub(cq, cm);
      const C od2 = mkc((T)0.5 * d2.y, (T)-0.5 * d2.x);
      tl[(kn)] = cadd(ev2, cmul(__ldg(&twy[kn]), od2));
    }
    tl[(k)] = xk;
  }
  __syncthreads();
  const int ntot = G * rows_out;
  const int lg = __ffs(G) - 1;  // G is a power of two
  for (int q = threadIdx.x; q < ntot; q += nthreads) {
    const int ky = q >> lg, g = q & (G - 1);
    vo[(size_t)ky * nx + ix0 + g] = sm[(size_t)g * lp + (ky)];
  }
}

// Asynchronous global -> shared copy of one complex element (cp.async, 8 or
// 16 bytes); when `live` is false the shared element is zero-filled and the
// source is not read.  cp_async_wait_all waits for this thread's copies;
// a block barrier then makes all of them visible.
template <typename C>
__device__ __forceinline__ void cp_async_elem(C* dst, const C* src, bool live) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = live ? (int)sizeof(C) : 0;
  if (sizeof(C) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---------------------------------------------------------------- y passes
// Shared memory of a y-pass block: G line regions of `lp` complex elements.
// A line region first holds the line's spectral column (index ky) and then
// serves as the line FFT's exchange buffer.  lp >= h + 1 and lp is chosen so
// that the G-wide column strips move without bank conflicts.

struct YJob {
  int zin;  // input Z array index
  int iky;  // multiply by i*ky before the transform (Dy, operators_par.c:110)
  int out;  // output physical field index
};

struct YInvArgs {
  Geo geo;
  const int* remaining; // batched launches: the member's step budget (0: skip the pass); nullptr: no budget
  int ycount;           // batched launches: blocks with blockIdx.y >= ycount have no work
  int lp;            // line pitch in shared memory (complex elements)
  const void* z;     // Z arrays (T2), stride (h+1)*nx
  int rows_in;       // Z rows that may be nonzero; the rest are read as zero
  const int* rows_dev;  // if set, overrides rows_in
  void* phys;        // physical arrays (T), stride nx*ny
  YJob jobs[MAX_JOBS];  // job of a block = jobs[blockIdx.y]
  // LEVEL: the block of job 0 (order-1 derivative of phi^(n+1)) also forms
  // W_n = job0 + sum_q phys[w_in[q]] * eta^(q+1) / (q+1)!
  // (hosm_2d_par.c:322-357 restated in physical space)
  int w_out;
  int eta;
  int w_terms;
  int w_in[MAX_TERMS];
  // LEVEL, fused with the next level's y-forward pass: the job-0 block also
  // forms P_(n+1) = -sum_p phys[nx_in[p-1]] eta^p/p! with the p = 1 term taken
  // from its own result (not stored), transforms it along y and writes V.
  int fuse_next;
  int nx_terms;
  int nx_in[MAX_TERMS];
  void* vout;
  int store_job0;  // 0 when the fused job-0 result has no other reader
  int plain_strip; // stage the column strip with loads and shared stores instead of cp.async
};

template <typename T, int H, int E, int MODE>
__device__ __forceinline__ void yinv_body(const YInvArgs& a, int bx, int by, int nthreads, const void* twv,
                                          const void* twyv, unsigned char* smraw) {
  using C = cpx<T>;
  constexpr int P = H / E;
  const C* tw = reinterpret_cast<const C*>(twv);    // length H
  const C* twy = reinterpret_cast<const C*>(twyv);  // length 2H
  const int G = nthreads / P;
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* sm = reinterpret_cast<C*>(smraw);
  C* tl = sm + (size_t)line * a.lp;
  const Geo& geo = a.geo;
  const int nx = geo.nx;
  const int ny = 2 * H;
  const int ix0 = bx * G;
  const int ix = ix0 + line;
  const size_t fsz = (size_t)(H + 1) * nx;
  const size_t psz = (size_t)nx * ny;
  const YJob J = a.jobs[by];
  T* pall = reinterpret_cast<T*>(a.phys);

  {  // column strip -> line regions; every row's copy is in flight at once
    const C* zs = reinterpret_cast<const C*>(a.z) + (size_t)J.zin * fsz;
    const int nin = G * (a.rows_dev ? *a.rows_dev : a.rows_in);
    const int ntot = G * (H + 1);
    const int lg = __ffs(G) - 1;  // G is a power of two
    if (a.plain_strip) {
      // every load in flight first, then the shared stores: an asynchronous
      // copy costs one shared-memory wavefront per 32-byte global sector,
      // these conflict-free stores one per 128 bytes.  A thread holds at
      // most ceil((H+1)/P) = E+1 elements.
      C buf[E + 1];
#pragma unroll
      for (int j = 0; j <= E; j++) {
        const int q = threadIdx.x + j * nthreads;
        buf[j] = q < nin ? __ldg(zs + (size_t)(q >> lg) * nx + ix0 + (q & (G - 1))) : mkc((T)0, (T)0);
      }
#pragma unroll
      for (int j = 0; j <= E; j++) {
        const int q = threadIdx.x + j * nthreads;
        if (q < ntot) sm[(size_t)(q & (G - 1)) * a.lp + (q >> lg)] = buf[j];
      }
    } else {
      for (int q = threadIdx.x; q < ntot; q += nthreads) {
        const int ky = q >> lg, g = q & (G - 1);
        const bool live = q < nin;
        cp_async_elem(&sm[(size_t)g * a.lp + ky], live ? zs + (size_t)ky * nx + ix0 + g : zs, live);
      }
      cp_async_wait_all();
    }
  }
  __syncthreads();
  // complex-to-real preprocessing: c[k] = Xe + i Xo (packing of a length-Ny
  // Hermitian sequence into a length-H complex one)
  C v[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int k = t + e * P;
    C A = tl[(k)];
    C Bv = tl[(H - k)];
    if (J.iky) {
      const T ka = ky_t<T>(geo, k), kb = ky_t<T>(geo, H - k);
      A = cscale(cmul_i(A), ka);
      Bv = cscale(cmul_i(Bv), kb);
    }
    if (k == 0) {  // FFTW c2r ignores Im of the ky = 0 and ky = Ny/2 bins
      A.y = (T)0;
      Bv.y = (T)0;
    }
    const C Bc = cconj(Bv);
    const C xe = cadd(A, Bc);
    const C d = csub(A, Bc);
    const C w = cconj(__ldg(&twy[k]));  // exp(+2 pi i k / Ny)
    v[e] = cadd(xe, cmul_i(cmul(d, w)));
  }
  line_fft<T, H, E, true>(v, tl, t, tw);  // starts with a barrier before reusing tl
  // v[e] holds (x[2m], x[2m+1]) for m = t + e*P of physical row ix
  C* po = reinterpret_cast<C*>(pall + (size_t)J.out * psz + (size_t)ix * ny);
  if (MODE != YI_LEVEL || by != 0 || a.store_job0) {
#pragma unroll
    for (int e = 0; e < E; e++) po[t + e * P] = v[e];
  }
  if (MODE == YI_LEVEL && by == 0) {
    // W_n = own + sum_{p=1..w_terms} d_p eta^p/p! with own = d_z phi^(n+1)
    // (this block's result) and w_in[q] the field of power q+1; then, when
    // fused, P_(n+1) = -(own eta + sum_{p=2..nx_terms} d'_p eta^p/p!).  Both
    // sums by Horner's rule from the highest power (acc = d_p + acc*eta/(p+1)).
    const C* pe = reinterpret_cast<const C*>(pall + (size_t)a.eta * psz + (size_t)ix * ny);
    C* pwo = reinterpret_cast<C*>(pall + (size_t)a.w_out * psz + (size_t)ix * ny);
    C et[E], acc[E];
#pragma unroll
    for (int e = 0; e < E; e++) et[e] = pe[t + e * P];
    {
      const C* pd = reinterpret_cast<const C*>(pall + (size_t)a.w_in[a.w_terms - 1] * psz + (size_t)ix * ny);
#pragma unroll
      for (int e = 0; e < E; e++) acc[e] = pd[t + e * P];
    }
    for (int q = a.w_terms - 2; q >= 0; q--) {
      const C* pd = reinterpret_cast<const C*>(pall + (size_t)a.w_in[q] * psz + (size_t)ix * ny);
      const T inv = (T)1 / (T)(q + 2);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const C d = pd[t + e * P];
        acc[e].x = d.x + acc[e].x * et[e].x * inv;
        acc[e].y = d.y + acc[e].y * et[e].y * inv;
      }
    }
#pragma unroll
    for (int e = 0; e < E; e++)
      pwo[t + e * P] = mkc(v[e].x + acc[e].x * et[e].x, v[e].y + acc[e].y * et[e].y);
    if (a.fuse_next) {
      // nx_in[q] holds the field of power q+1 for q >= 1; power 1 is own
      if (a.nx_terms > 1) {
        const C* pd = reinterpret_cast<const C*>(pall + (size_t)a.nx_in[a.nx_terms - 1] * psz + (size_t)ix * ny);
#pragma unroll
        for (int e = 0; e < E; e++) acc[e] = pd[t + e * P];
        for (int q = a.nx_terms - 2; q >= 1; q--) {
          const C* pq = reinterpret_cast<const C*>(pall + (size_t)a.nx_in[q] * psz + (size_t)ix * ny);
          const T inv = (T)1 / (T)(q + 2);
#pragma unroll
          for (int e = 0; e < E; e++) {
            const C d = pq[t + e * P];
            acc[e].x = d.x + acc[e].x * et[e].x * inv;
            acc[e].y = d.y + acc[e].y * et[e].y * inv;
          }
        }
#pragma unroll
        for (int e = 0; e < E; e++) {
          acc[e].x = v[e].x + acc[e].x * et[e].x * (T)0.5;
          acc[e].y = v[e].y + acc[e].y * et[e].y * (T)0.5;
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; e++) acc[e] = v[e];
      }
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = mkc(-acc[e].x * et[e].x, -acc[e].y * et[e].y);
    }
  }
  if (MODE == YI_LEVEL && a.fuse_next && by == 0)
    yfwd_finish<T, H, E>(v, sm, tl, t, G, a.lp, tw, twy, reinterpret_cast<C*>(a.vout), nx, ix0, H + 1, nthreads);
}

template <typename T, int H, int E, int MODE, bool B>
__global__ void __launch_bounds__(MAX_THREADS, 2) k_yinv(const __grid_constant__ YInvArgs a0,
                                                         const YInvArgs* __restrict__ arr, const void* twv,
                                                         const void* twyv) {
  pdl_enter();
  const YInvArgs& a = B ? arr[blockIdx.z] : a0;
  if (B && (int)blockIdx.y >= a.ycount) return;
  if (B && a.remaining && *a.remaining == 0) return;  // the member's step budget is spent
  extern __shared__ __align__(16) unsigned char smraw[];
  yinv_body<T, H, E, MODE>(a, blockIdx.x, blockIdx.y, blockDim.x, twv, twyv, smraw);
}

struct YFwdArgs {
  Geo geo;
  const int* remaining; // batched launches: the member's step budget (0: skip the pass); nullptr: no budget
  int ycount;           // batched launches: blocks with blockIdx.y >= ycount have no work
  int lp;
  const void* phys;   // physical arrays (T), stride nx*ny
  const void* in_ptr; // PLAIN: physical input (T) [nx][ny]
  // LEVEL: P = -sum_q phys[t_in[q]] * eta^(q+1) / (q+1)!  (hosm_2d_par.c:302-317)
  int eta;
  int nterms;
  int t_in[MAX_TERMS];
  // RHS (blockIdx.y = 0: P_eta, 1: P_phi)
  int ex, ey, px, py;
  int L;
  int w_idx[MAX_TERMS];  // W_0..W_L
  int which_base;        // RHS: output blockIdx.y computes quantity which_base + blockIdx.y
  void* vout;            // output V arrays (T2), stride (h+1)*nx; output = blockIdx.y
  int rows_out;
};

// RHS assembly at one physical point: P_eta (which = 0) or P_phi (which = 1);
// which = 2..5 give the physical parts of Zvel's outputs: W^(M) and W^(M-2)
// without W^(1) (which is added in spectral space), (W^2)^(M), (W^2)^(M-2)
// (hosm_2d_par.c:362-442).
template <typename T>
__device__ __forceinline__ T rhs_point(const YFwdArgs& a, const T* W, T ex, T ey, T px, T py, int which) {
  const int L = a.L;
  const T grad2 = ex * ex + ey * ey;
  if (which == 2 || which == 3) {
    T s = (T)0;
#pragma unroll
    for (int n = 1; n < MAX_TERMS; n++)
      if (n <= (which == 2 ? L : L - 2)) s += W[n];
    return s;
  }
  if (which == 0) {
    T s1 = (T)0, wm2 = (T)0;
#pragma unroll
    for (int n = 0; n < MAX_TERMS; n++) {
      if (n >= 1 && n <= L) s1 += W[n];
      if (n <= L - 2) wm2 += W[n];
    }
    return -(ex * px + ey * py) + s1 + grad2 * wm2;  // hosm_2d_par.c:150-176
  }
  // W2M2 = sum_{n<=L-3} sum_m W_m W_{n-m};  W2M = W2M2 + sum_{n=L-2}^{L-1} ...  (hosm_2d_par.c:397-442)
  T w2m2 = (T)0, w2m = (T)0;
#pragma unroll
  for (int n = 0; n < MAX_TERMS; n++) {
    if (n > L - 1) continue;
    T s = (T)0;
#pragma unroll
    for (int m = 0; m <= n; m++) s += W[m] * W[n - m];
    if (n <= L - 3) w2m2 += s;
    else w2m += s;
  }
  w2m += w2m2;
  if (which == 4) return w2m;
  if (which == 5) return w2m2;
  return (T)0.5 * (w2m + grad2 * w2m2) - (T)0.5 * (px * px + py * py);  // hosm_2d_par.c:181-206
}

template <typename T, int H, int E, int MODE>
__device__ __forceinline__ void yfwd_body(const YFwdArgs& a, int bx, int by, int nthreads, const void* twv,
                                          const void* twyv, unsigned char* smraw) {
  using C = cpx<T>;
  constexpr int P = H / E;
  const C* tw = reinterpret_cast<const C*>(twv);
  const C* twy = reinterpret_cast<const C*>(twyv);
  const int G = nthreads / P;
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* sm = reinterpret_cast<C*>(smraw);
  C* tl = sm + (size_t)line * a.lp;
  const Geo& geo = a.geo;
  const int nx = geo.nx;
  const int ny = 2 * H;
  const int ix0 = bx * G;
  const int ix = ix0 + line;
  const size_t fsz = (size_t)(H + 1) * nx;
  const size_t psz = (size_t)nx * ny;
  const T* pall = reinterpret_cast<const T*>(a.phys);
  const size_t rowoff = (size_t)ix * ny;

  C v[E];
  if (MODE == YF_PLAIN) {
    const C* src = reinterpret_cast<const C*>(reinterpret_cast<const T*>(a.in_ptr) + rowoff);
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[t + e * P];
  } else if (MODE == YF_LEVEL) {
    // P = -sum_{p=1..nterms} d_p eta^p/p! (t_in[q] holds the field of power
    // q+1), by Horner's rule from the highest power: acc = d_n, acc = d_p +
    // acc*eta/(p+1) down to p = 1, P = -acc*eta
    const C* pe = reinterpret_cast<const C*>(pall + (size_t)a.eta * psz + rowoff);
    C et[E];
#pragma unroll
    for (int e = 0; e < E; e++) et[e] = pe[t + e * P];
    {
      const C* pd = reinterpret_cast<const C*>(pall + (size_t)a.t_in[a.nterms - 1] * psz + rowoff);
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = pd[t + e * P];
    }
    for (int q = a.nterms - 2; q >= 0; q--) {
      const C* pd = reinterpret_cast<const C*>(pall + (size_t)a.t_in[q] * psz + rowoff);
      const T inv = (T)1 / (T)(q + 2);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const C d = pd[t + e * P];
        v[e].x = d.x + v[e].x * et[e].x * inv;
        v[e].y = d.y + v[e].y * et[e].y * inv;
      }
    }
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = mkc(-v[e].x * et[e].x, -v[e].y * et[e].y);
  } else {
    const int which = by + a.which_base;
    const C* pex = reinterpret_cast<const C*>(pall + (size_t)a.ex * psz + rowoff);
    const C* pey = reinterpret_cast<const C*>(pall + (size_t)a.ey * psz + rowoff);
    const C* ppx = reinterpret_cast<const C*>(pall + (size_t)a.px * psz + rowoff);
    const C* ppy = reinterpret_cast<const C*>(pall + (size_t)a.py * psz + rowoff);
    const int L = a.L;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int m = t + e * P;
      const C ex = pex[m], ey = pey[m], px = ppx[m], py = ppy[m];
      T W0[MAX_TERMS], W1[MAX_TERMS];
#pragma unroll
      for (int n = 0; n < MAX_TERMS; n++) {
        C w = mkc((T)0, (T)0);
        if (n <= L) w = reinterpret_cast<const C*>(pall + (size_t)a.w_idx[n] * psz + rowoff)[m];
        W0[n] = w.x;
        W1[n] = w.y;
      }
      v[e] = mkc(rhs_point<T>(a, W0, ex.x, ey.x, px.x, py.x, which), rhs_point<T>(a, W1, ex.y, ey.y, px.y, py.y, which));
    }
  }

  yfwd_finish<T, H, E>(v, sm, tl, t, G, a.lp, tw, twy, reinterpret_cast<C*>(a.vout) + (size_t)by * fsz, nx, ix0,
                       a.rows_out, nthreads);
}

template <typename T, int H, int E, int MODE, bool B>
__global__ void __launch_bounds__(MAX_THREADS, 2) k_yfwd(const __grid_constant__ YFwdArgs a0,
                                                         const YFwdArgs* __restrict__ arr, const void* twv,
                                                         const void* twyv) {
  pdl_enter();
  const YFwdArgs& a = B ? arr[blockIdx.z] : a0;
  if (B && (int)blockIdx.y >= a.ycount) return;
  if (B && a.remaining && *a.remaining == 0) return;  // the member's step budget is spent
  extern __shared__ __align__(16) unsigned char smraw[];
  yfwd_body<T, H, E, MODE>(a, blockIdx.x, blockIdx.y, blockDim.x, twv, twyv, smraw);
}

// ---------------------------------------------------------------- step end
// Sums the stage-0 Hamiltonian partials (one per ky row) in a fixed order
// (fixed strides, fixed tree), records (t, H) and advances t
// (time_schemes_par.c:73-93,119).  One block of nthreads (a power of two,
// at most 256) threads.
struct StepEndArgs {
  const double* ham_part;
  int nparts;
  double* tdev;
  double dt;
  long long* stepdev;
  double* ham_hist;
  double* t_hist;
  int hist_cap;
  long long* bad_step;  // first step whose energy was not finite (-1: none)
  int* any_bad;         // ensemble-wide word set with bad_step (nullptr outside ensembles)
  int* remaining;       // the member's step budget, counted down here (nullptr: none)
};

__device__ __forceinline__ void step_end_body(const StepEndArgs& a, int nthreads) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < a.nparts; i += nthreads) s += a.ham_part[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = nthreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const long long st = *a.stepdev;
  if (st >= 0) {  // ring of hist_cap records
    a.ham_hist[st % a.hist_cap] = red[0];
    a.t_hist[st % a.hist_cap] = *a.tdev;
  }
  // the energy sums every mode of eta and phi, so a NaN or Inf anywhere in the
  // state shows here; the host reads this word at hos_sync
  if (!isfinite(red[0])) {
    if (*a.bad_step < 0) *a.bad_step = st;
    if (a.any_bad) *a.any_bad = 1;
  }
  *a.tdev = *a.tdev + a.dt;
  *a.stepdev = st + 1;
  if (a.remaining && *a.remaining > 0) *a.remaining = *a.remaining - 1;
}

}  // namespace hos
