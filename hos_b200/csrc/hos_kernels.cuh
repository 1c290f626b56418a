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
// or written as G-wide column strips staged through a shared-memory tile.
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
__device__ __forceinline__ double dz_mult(double kz, double th, int p) {
  double m = 1.0;
  for (int q = 0; q < p; q++) m *= kz;
  return (p & 1) ? m * th : m;
}

// ---------------------------------------------------------------- x inverse
struct XInvArgs {
  Geo geo;
  int mode;  // 0: RK stage (4 + ndz outputs); 1: plain c2r x-pass of one field
  int rows;  // ky rows that may be nonzero in the input
  const int* rows_dev;  // if set, overrides rows (active rows of the state, kept on the device)
  const double2* u;                 // stage: packed state [2][h+1][nx]; plain: one field
  const double2* kp[MAX_STAGES];    // earlier stage derivatives
  double coef[MAX_STAGES];          // dt*b[s][p]
  int nk;
  int ndz;                          // number of z-derivative outputs (orders 1..ndz)
  void* z;                          // output complex arrays, stride (h+1)*nx
  const double* tdev;               // simulation time (device)
  double* rdev;                     // ramp factor for this step (device), written if set_ramp
  int set_ramp;
  double tramp;
  int rampflg;
};

template <typename T, int NX, int E>
__global__ void __launch_bounds__(MAX_THREADS) k_xinv(const __grid_constant__ XInvArgs a, const void* twv) {
  using C = cpx<T>;
  constexpr int P = NX / E;
  const C* tw = reinterpret_cast<const C*>(twv);
  extern __shared__ __align__(16) unsigned char smraw[];
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* sm = reinterpret_cast<C*>(smraw) + line * line_smem_elems<NX, E>();
  const int lines = blockDim.x / P;
  const int row = blockIdx.x * lines + line;
  const int rows = a.rows_dev ? *a.rows_dev : a.rows;
  const bool live = row < rows;
  const Geo& geo = a.geo;
  const size_t fsz = (size_t)(geo.h + 1) * NX;
  const size_t roff = (size_t)(live ? row : 0) * NX;
  C* z = reinterpret_cast<C*>(a.z);

  if (a.set_ramp && blockIdx.x == 0 && threadIdx.x == 0) {
    double r = 1.0;
    if (a.rampflg == 1) {
      const double tt = *a.tdev;
      r = 1 - exp(-tt * tt / a.tramp / a.tramp);  // RampFun, hosm_2d_par.c:526-530
    }
    *a.rdev = r;
  }
  if ((int)(blockIdx.x * lines) >= rows) return;  // whole block beyond the active rows

  C v[E];
  if (a.mode == 1) {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = live ? conv<T>(a.u[roff + t + e * P]) : mkc((T)0, (T)0);
    line_fft<T, NX, E, true>(v, sm, t, tw);
    if (live) {
#pragma unroll
      for (int e = 0; e < E; e++) z[roff + t + e * P] = v[e];
    }
    return;
  }

  const double ky = ky_of(geo, row);
  double2 w[E];
  // ---- eta: stage input (time_schemes_par.c:38-67)
#pragma unroll
  for (int e = 0; e < E; e++) {
    double2 x = make_double2(0.0, 0.0);
    if (live) {
      const size_t idx = roff + t + e * P;
      x = a.u[idx];
      for (int p = 0; p < a.nk; p++) {
        const double2 kk = a.kp[p][idx];
        x.x = x.x + a.coef[p] * kk.x;
        x.y = x.y + a.coef[p] * kk.y;
      }
    }
    w[e] = x;
  }
  // out 0: eta
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = conv<T>(w[e]);
  line_fft<T, NX, E, true>(v, sm, t, tw);
  if (live) {
#pragma unroll
    for (int e = 0; e < E; e++) z[roff + t + e * P] = v[e];
  }
  // out 1: i kx eta (Dx, operators_par.c:66)
#pragma unroll
  for (int e = 0; e < E; e++) {
    const double kx = kx_of(geo, t + e * P);
    v[e] = conv<T>(make_double2(-kx * w[e].y, kx * w[e].x));
  }
  line_fft<T, NX, E, true>(v, sm, t, tw);
  if (live) {
#pragma unroll
    for (int e = 0; e < E; e++) z[fsz + roff + t + e * P] = v[e];
  }
  // ---- phi stage input
#pragma unroll
  for (int e = 0; e < E; e++) {
    double2 x = make_double2(0.0, 0.0);
    if (live) {
      const size_t idx = fsz + roff + t + e * P;
      x = a.u[idx];
      for (int p = 0; p < a.nk; p++) {
        const double2 kk = a.kp[p][idx];
        x.x = x.x + a.coef[p] * kk.x;
        x.y = x.y + a.coef[p] * kk.y;
      }
    }
    w[e] = x;
  }
  // out 2: phi (its y-derivative is taken in the y-pass)
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = conv<T>(w[e]);
  line_fft<T, NX, E, true>(v, sm, t, tw);
  if (live) {
#pragma unroll
    for (int e = 0; e < E; e++) z[2 * fsz + roff + t + e * P] = v[e];
  }
  // out 3: i kx phi
#pragma unroll
  for (int e = 0; e < E; e++) {
    const double kx = kx_of(geo, t + e * P);
    v[e] = conv<T>(make_double2(-kx * w[e].y, kx * w[e].x));
  }
  line_fft<T, NX, E, true>(v, sm, t, tw);
  if (live) {
#pragma unroll
    for (int e = 0; e < E; e++) z[3 * fsz + roff + t + e * P] = v[e];
  }
  // out 4..: z-derivatives of phi of orders 1..ndz (Dz, operators_par.c:168-192)
  double kz[E], th[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const double kx = kx_of(geo, t + e * P);
    kz[e] = sqrt(kx * kx + ky * ky);
    th[e] = geo.depth > 0 ? tanh(kz[e] * geo.depth) : 1.0;
  }
  for (int p = 1; p <= a.ndz; p++) {
#pragma unroll
    for (int e = 0; e < E; e++) {
      const double m = dz_mult(kz[e], th[e], p);
      v[e] = conv<T>(make_double2(m * w[e].x, m * w[e].y));
    }
    line_fft<T, NX, E, true>(v, sm, t, tw);
    if (live) {
#pragma unroll
      for (int e = 0; e < E; e++) z[(size_t)(3 + p) * fsz + roff + t + e * P] = v[e];
    }
  }
}

// ---------------------------------------------------------------- x forward
struct XFwdArgs {
  Geo geo;
  int mode;       // 0: plain r2c x-pass -> FP64 spectral; 1: level (forward, then ndz inverse outputs); 2: RK stage end
  int rows;       // rows processed
  const int* rows_dev;  // if set, overrides rows
  int rows_fft;   // mode 2: rows < rows_fft are transformed; rows in [rows_fft, rows) only add to the Hamiltonian
  const void* vin0;  // input V arrays (T2) [h+1][nx]
  const void* vin1;
  double2* out_spec;  // mode 0 output
  int dealias;        // mode 0: zero the modes Dealias zeroes (operators_par.c:283-325)
  void* zout;         // mode 1: output Z arrays (T2), stride (h+1)*nx
  int ndz;
  // mode 2
  const double2* u;               // packed state at step start (updated in place on the final stage)
  const double2* kp[MAX_STAGES];  // earlier stage derivatives (stage input = u + sum coef*kp)
  double coef[MAX_STAGES];
  int nk;
  double2* kout;                  // this stage's derivative [2][h+1][nx]
  const double* rdev;             // ramp factor
  int ham;                        // accumulate the stage-0 Hamiltonian
  double* ham_part;               // one partial per block
  int final_update;               // u += sum cfin[s] * k_s (time_schemes_par.c:98-116)
  const double2* kall[MAX_STAGES];
  double cfin[MAX_STAGES];
  int nstage;                     // number of stages; k of the last one is in registers
  double2* unew;
};

template <typename T, int NX, int E>
__global__ void __launch_bounds__(MAX_THREADS) k_xfwd(const __grid_constant__ XFwdArgs a, const void* twv) {
  using C = cpx<T>;
  constexpr int P = NX / E;
  const C* tw = reinterpret_cast<const C*>(twv);
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[MAX_THREADS / 32];
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* sm = reinterpret_cast<C*>(smraw) + line * line_smem_elems<NX, E>();
  const int lines = blockDim.x / P;
  const int row = blockIdx.x * lines + line;
  const Geo& geo = a.geo;
  const size_t fsz = (size_t)(geo.h + 1) * NX;
  const T sc = (T)geo.inv_nxny;

  if (a.mode != 2) {
    const bool live = row < a.rows;
    const size_t roff = (size_t)(live ? row : 0) * NX;
    const C* vin = reinterpret_cast<const C*>(a.vin0);
    C v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = live ? vin[roff + t + e * P] : mkc((T)0, (T)0);
    line_fft<T, NX, E, false>(v, sm, t, tw);
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = cscale(v[e], sc);  // fft_2d's 1/Nx/Ny (exact: powers of two)
    if (a.mode == 0) {
      if (live) {
#pragma unroll
        for (int e = 0; e < E; e++) {
          const bool z0 = a.dealias && !keep_mode(geo, t + e * P, row);
          a.out_spec[roff + t + e * P] = z0 ? make_double2(0.0, 0.0) : widen(v[e]);
        }
      }
      return;
    }
    // mode 1: phi^(n+1) hat is in v; emit its z-derivatives of orders 1..ndz
    const double ky = ky_of(geo, row);
    double kz[E], th[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const double kx = kx_of(geo, t + e * P);
      kz[e] = sqrt(kx * kx + ky * ky);
      th[e] = geo.depth > 0 ? tanh(kz[e] * geo.depth) : 1.0;
    }
    C* z = reinterpret_cast<C*>(a.zout);
    for (int p = 1; p <= a.ndz; p++) {
      C w[E];
#pragma unroll
      for (int e = 0; e < E; e++) w[e] = cscale(v[e], (T)dz_mult(kz[e], th[e], p));
      line_fft<T, NX, E, true>(w, sm, t, tw);
      if (live) {
#pragma unroll
        for (int e = 0; e < E; e++) z[(size_t)(p - 1) * fsz + roff + t + e * P] = w[e];
      }
    }
    return;
  }

  // ---- mode 2: end of an RK stage (rhs_hos tail, hosm_2d_par.c:181-233, and
  // sol_update_RK bookkeeping, time_schemes_par.c:70-116)
  const int rows = a.rows_dev ? *a.rows_dev : a.rows;
  const bool live = row < rows;
  const bool fft_row = row < a.rows_fft;
  const size_t roff = (size_t)(live ? row : 0) * NX;
  const bool block_fft = (int)(blockIdx.x * lines) < a.rows_fft;
  double2 se[E], sp[E];
  if (block_fft) {
    const C* v0 = reinterpret_cast<const C*>(a.vin0);
    const C* v1 = reinterpret_cast<const C*>(a.vin1);
    C v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = fft_row ? v0[roff + t + e * P] : mkc((T)0, (T)0);
    line_fft<T, NX, E, false>(v, sm, t, tw);
#pragma unroll
    for (int e = 0; e < E; e++) se[e] = widen(cscale(v[e], sc));
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = fft_row ? v1[roff + t + e * P] : mkc((T)0, (T)0);
    line_fft<T, NX, E, false>(v, sm, t, tw);
#pragma unroll
    for (int e = 0; e < E; e++) sp[e] = widen(cscale(v[e], sc));
  } else {
#pragma unroll
    for (int e = 0; e < E; e++) {
      se[e] = make_double2(0.0, 0.0);
      sp[e] = make_double2(0.0, 0.0);
    }
  }
  double hacc = 0.0;
  if (live) {
    const double ky = ky_of(geo, row);
    const double R = *a.rdev;
    const double wrow = (row == 0) ? 1.0 : 2.0;  // Hamiltonian weights, hosm_2d_par.c:473-519
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int i = t + e * P;
      const size_t idx = roff + i;
      double2 ue = a.u[idx], up = a.u[fsz + idx];
      const double2 u0e = ue, u0p = up;
      for (int p = 0; p < a.nk; p++) {
        const double2 k0 = a.kp[p][idx], k1 = a.kp[p][fsz + idx];
        ue.x = ue.x + a.coef[p] * k0.x;
        ue.y = ue.y + a.coef[p] * k0.y;
        up.x = up.x + a.coef[p] * k1.x;
        up.y = up.y + a.coef[p] * k1.y;
      }
      double2 et = make_double2(0.0, 0.0), pt = make_double2(0.0, 0.0);
      if (fft_row && keep_mode(geo, i, row)) {
        const double kx = kx_of(geo, i);
        const double kz = sqrt(kx * kx + ky * ky);
        const double m1 = dz_mult(kz, geo.depth > 0 ? tanh(kz * geo.depth) : 1.0, 1);
        // eta_t = R * NL_eta + Dz phi ; phi_t = R * NL_phi - g eta  (R = 1 without ramp)
        et.x = R * se[e].x + m1 * up.x;
        et.y = R * se[e].y + m1 * up.y;
        pt.x = R * sp[e].x - geo.g * ue.x;
        pt.y = R * sp[e].y - geo.g * ue.y;
      }
      if (fft_row) {
        a.kout[idx] = et;
        a.kout[fsz + idx] = pt;
      }
      if (a.ham) {
        hacc += wrow * (geo.g * u0e.x * u0e.x + geo.g * u0e.y * u0e.y + u0p.x * et.x + u0p.y * et.y);
      }
      if (a.final_update && fft_row) {
        double2 ne = u0e, np = u0p;
        for (int s = 0; s + 1 < a.nstage; s++) {
          const double2 k0 = a.kall[s][idx], k1 = a.kall[s][fsz + idx];
          ne.x = ne.x + a.cfin[s] * k0.x;
          ne.y = ne.y + a.cfin[s] * k0.y;
          np.x = np.x + a.cfin[s] * k1.x;
          np.y = np.y + a.cfin[s] * k1.y;
        }
        const double cl = a.cfin[a.nstage - 1];
        ne.x = ne.x + cl * et.x;
        ne.y = ne.y + cl * et.y;
        np.x = np.x + cl * pt.x;
        np.y = np.y + cl * pt.y;
        a.unew[idx] = ne;
        a.unew[fsz + idx] = np;
      }
    }
  }
  if (a.ham) {
    // deterministic block reduction
    for (int o = 16; o > 0; o >>= 1) hacc += __shfl_down_sync(0xffffffffu, hacc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = hacc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int wi = 0; wi < (int)(blockDim.x + 31) / 32; wi++) s += red[wi];
      a.ham_part[blockIdx.x] = s;
    }
  }
}

// ---------------------------------------------------------------- y inverse
struct YJob {
  int zin;  // input Z array index
  int iky;  // multiply by i*ky before the transform (Dy, operators_par.c:110)
  int out;  // output physical field index
};

struct YInvArgs {
  Geo geo;
  int tp;            // tile pitch (complex elements per line)
  const void* z;     // Z arrays (T2), stride (h+1)*nx
  int rows_in;       // Z rows that may be nonzero; the rest are read as zero
  const int* rows_dev;  // if set, overrides rows_in
  void* phys;        // physical arrays (T), stride nx*ny
  int njobs;
  YJob jobs[MAX_JOBS];
  // W_n epilogue on job 0 (hosm_2d_par.c:322-357 restated in physical space):
  // W = job0 + sum_m phys[w_in[m]] * eta^w_pow[m] / w_pow[m]!
  int wmode;
  int w_out;
  int eta;
  int w_terms;
  int w_in[MAX_TERMS];
  int w_pow[MAX_TERMS];
};

template <typename T, int H, int E>
__global__ void __launch_bounds__(MAX_THREADS) k_yinv(const __grid_constant__ YInvArgs a, const void* twv) {
  using C = cpx<T>;
  constexpr int P = H / E;
  const C* tw = reinterpret_cast<const C*>(twv);
  extern __shared__ __align__(16) unsigned char smraw[];
  const int G = blockDim.x / P;
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* tile = reinterpret_cast<C*>(smraw);
  C* xb = tile + (size_t)G * a.tp + line * line_smem_elems<H, E>();
  C* tl = tile + (size_t)line * a.tp;
  const Geo& geo = a.geo;
  const int nx = geo.nx;
  const int ix0 = blockIdx.x * G;
  const int ix = ix0 + line;
  const size_t fsz = (size_t)(H + 1) * nx;
  const size_t psz = (size_t)nx * (2 * H);
  const C* zall = reinterpret_cast<const C*>(a.z);
  T* pall = reinterpret_cast<T*>(a.phys);
  const int ny = 2 * H;
  const int tws = TW_N / ny;

  int cur = -1;
  for (int jb = 0; jb < a.njobs; jb++) {
    const YJob J = a.jobs[jb];
    if (J.zin != cur) {
      __syncthreads();
      const C* zs = zall + (size_t)J.zin * fsz;
      const int nin = G * (a.rows_dev ? *a.rows_dev : a.rows_in);
      const int ntot = G * (H + 1);
      for (int q = threadIdx.x; q < ntot; q += blockDim.x) {
        const int ky = q / G, g = q - ky * G;
        tile[(size_t)g * a.tp + ky] = (q < nin) ? zs[(size_t)ky * nx + ix0 + g] : mkc((T)0, (T)0);
      }
      __syncthreads();
      cur = J.zin;
    }
    // complex-to-real preprocessing: c[k] = Xe + i Xo (packing of a length-Ny
    // Hermitian sequence into a length-H complex one)
    C v[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int k = t + e * P;
      C A = tl[k];
      C B = tl[H - k];
      if (J.iky) {
        const T ka = (T)ky_of(geo, k), kb = (T)ky_of(geo, H - k);
        A = cscale(cmul_i(A), ka);
        B = cscale(cmul_i(B), kb);
      }
      if (k == 0) {  // FFTW c2r ignores Im of the ky = 0 and ky = Ny/2 bins
        A.y = (T)0;
        B.y = (T)0;
      }
      const C Bc = cconj(B);
      const C xe = cadd(A, Bc);
      const C d = csub(A, Bc);
      const C w = cconj(__ldg(&tw[k * tws]));  // exp(+2 pi i k / Ny)
      const C xo = cmul(d, w);
      v[e] = cadd(xe, cmul_i(xo));
    }
    line_fft<T, H, E, true>(v, xb, t, tw);
    // v[e] holds (x[2m], x[2m+1]) for m = t + e*P of physical row ix
    C* po = reinterpret_cast<C*>(pall + (size_t)J.out * psz + (size_t)ix * ny);
#pragma unroll
    for (int e = 0; e < E; e++) po[t + e * P] = v[e];
    if (a.wmode && jb == 0) {
      const C* pe = reinterpret_cast<const C*>(pall + (size_t)a.eta * psz + (size_t)ix * ny);
      C* pw = reinterpret_cast<C*>(pall + (size_t)a.w_out * psz + (size_t)ix * ny);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int m = t + e * P;
        const C et = pe[m];
        C acc = mkc((T)0, (T)0);
        for (int q = 0; q < a.w_terms; q++) {
          const C d = reinterpret_cast<const C*>(pall + (size_t)a.w_in[q] * psz + (size_t)ix * ny)[m];
          T px = (T)1, py = (T)1, f = (T)1;
          for (int r = 1; r <= a.w_pow[q]; r++) {
            px *= et.x;
            py *= et.y;
            f *= (T)r;
          }
          acc.x += d.x * px / f;
          acc.y += d.y * py / f;
        }
        acc.x += v[e].x;
        acc.y += v[e].y;
        pw[m] = acc;
      }
    }
  }
}

// ---------------------------------------------------------------- y forward
struct YFwdArgs {
  Geo geo;
  int tp;
  int mode;           // 0: plain (field in0); 1: Taylor level P_n; 2: RHS assembly (P_eta, P_phi)
  const void* phys;   // physical arrays (T), stride nx*ny
  const void* in_ptr; // mode 0: physical input (T) [nx][ny]
  // mode 1: P = -sum_q phys[t_in[q]] * eta^t_pow[q] / t_pow[q]!  (hosm_2d_par.c:302-317)
  int eta;
  int nterms;
  int t_in[MAX_TERMS];
  int t_pow[MAX_TERMS];
  // mode 2
  int ex, ey, px, py;
  int L;
  int w_idx[MAX_TERMS];  // W_0..W_L
  void* vout;            // output V arrays (T2), stride (h+1)*nx
  int rows_out;
};

template <typename T>
__device__ __forceinline__ void rhs_point(const YFwdArgs& a, const T* const* Wp, size_t off, T ex, T ey, T px, T py,
                                          T& pe, T& pp) {
  T W[MAX_TERMS];
  const int L = a.L;
#pragma unroll
  for (int n = 0; n < MAX_TERMS; n++) W[n] = (n <= L) ? Wp[n][off] : (T)0;
  const T grad2 = ex * ex + ey * ey;
  T s1 = (T)0, wm2 = (T)0;
#pragma unroll
  for (int n = 0; n < MAX_TERMS; n++) {
    if (n >= 1 && n <= L) s1 += W[n];
    if (n <= L - 2) wm2 += W[n];
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
  pe = -(ex * px + ey * py) + s1 + grad2 * wm2;                        // hosm_2d_par.c:150-176
  pp = (T)0.5 * (w2m + grad2 * w2m2) - (T)0.5 * (px * px + py * py);  // hosm_2d_par.c:181-206
}

template <typename T, int H, int E>
__global__ void __launch_bounds__(MAX_THREADS) k_yfwd(const __grid_constant__ YFwdArgs a, const void* twv) {
  using C = cpx<T>;
  constexpr int P = H / E;
  const C* tw = reinterpret_cast<const C*>(twv);
  extern __shared__ __align__(16) unsigned char smraw[];
  const int G = blockDim.x / P;
  const int line = threadIdx.x / P;
  const int t = threadIdx.x - line * P;
  C* tile = reinterpret_cast<C*>(smraw);
  C* xb = tile + (size_t)G * a.tp + line * line_smem_elems<H, E>();
  C* tl = tile + (size_t)line * a.tp;
  const Geo& geo = a.geo;
  const int nx = geo.nx;
  const int ny = 2 * H;
  const int ix0 = blockIdx.x * G;
  const int ix = ix0 + line;
  const size_t fsz = (size_t)(H + 1) * nx;
  const size_t psz = (size_t)nx * ny;
  const T* pall = reinterpret_cast<const T*>(a.phys);
  const size_t rowoff = (size_t)ix * ny;
  C* vall = reinterpret_cast<C*>(a.vout);
  const int tws = TW_N / ny;
  const int nout = (a.mode == 2) ? 2 : 1;

  C v[E], v2[E];
  if (a.mode == 0) {
    const C* src = reinterpret_cast<const C*>(reinterpret_cast<const T*>(a.in_ptr) + rowoff);
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[t + e * P];
  } else if (a.mode == 1) {
    const C* pe = reinterpret_cast<const C*>(pall + (size_t)a.eta * psz + rowoff);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int m = t + e * P;
      const C et = pe[m];
      C acc = mkc((T)0, (T)0);
      for (int q = 0; q < a.nterms; q++) {
        const C d = reinterpret_cast<const C*>(pall + (size_t)a.t_in[q] * psz + rowoff)[m];
        T px = (T)1, py = (T)1, f = (T)1;
        for (int r = 1; r <= a.t_pow[q]; r++) {
          px *= et.x;
          py *= et.y;
          f *= (T)r;
        }
        acc.x -= d.x * px / f;
        acc.y -= d.y * py / f;
      }
      v[e] = acc;
    }
  } else {
    const T* Wp[MAX_TERMS];
#pragma unroll
    for (int n = 0; n < MAX_TERMS; n++) Wp[n] = pall + (size_t)a.w_idx[n < a.L + 1 ? n : 0] * psz + rowoff;
    const T* pex = pall + (size_t)a.ex * psz + rowoff;
    const T* pey = pall + (size_t)a.ey * psz + rowoff;
    const T* ppx = pall + (size_t)a.px * psz + rowoff;
    const T* ppy = pall + (size_t)a.py * psz + rowoff;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int m = t + e * P;
      T pe0, pp0, pe1, pp1;
      rhs_point<T>(a, Wp, 2 * m, pex[2 * m], pey[2 * m], ppx[2 * m], ppy[2 * m], pe0, pp0);
      rhs_point<T>(a, Wp, 2 * m + 1, pex[2 * m + 1], pey[2 * m + 1], ppx[2 * m + 1], ppy[2 * m + 1], pe1, pp1);
      v[e] = mkc(pe0, pe1);
      v2[e] = mkc(pp0, pp1);
    }
  }

  for (int o = 0; o < nout; o++) {
    if (o == 1) {
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = v2[e];
    }
    line_fft<T, H, E, false>(v, xb, t, tw);
    // C[k] natural order -> shared buffer, then real-to-complex postprocessing
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; e++) xb[spad<E>(t + e * P)] = v[e];
    __syncthreads();
#pragma unroll
    for (int e = 0; e <= E; e++) {
      int k;
      if (e < E) k = t + e * P;
      else if (t == 0) k = H;
      else break;
      const C ck = xb[spad<E>(k & (H - 1))];
      const C cn = cconj(xb[spad<E>((H - k) & (H - 1))]);
      const C ev = cscale(cadd(ck, cn), (T)0.5);
      const C d = csub(ck, cn);
      const C od = mkc((T)0.5 * d.y, (T)-0.5 * d.x);  // (ck - cn) / (2i)
      const C w = __ldg(&tw[k * tws]);              // exp(-2 pi i k / Ny)
      tl[k] = cadd(ev, cmul(w, od));
    }
    __syncthreads();
    C* vo = vall + (size_t)o * fsz;
    const int ntot = G * a.rows_out;
    for (int q = threadIdx.x; q < ntot; q += blockDim.x) {
      const int ky = q / G, g = q - ky * G;
      vo[(size_t)ky * nx + ix0 + g] = tile[(size_t)g * a.tp + ky];
    }
  }
}

}  // namespace hos
