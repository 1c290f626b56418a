// Shared-memory Stockham line FFT for sm_100a.
//
// A "line" is one 1-D complex sequence of length N (a power of two).  P = N/E
// threads cooperate on a line and each keeps E elements in registers.  On
// entry and on exit thread t holds element t + e*P in register e, so the
// first radix pass reads and the last radix pass writes global memory with
// consecutive threads on consecutive addresses.  Radix-E butterflies run in
// registers; between passes the line is exchanged through a padded
// shared-memory buffer.
//
// The pass structure is the Stockham autosort formulation of Govindaraju et
// al., "High Performance Discrete Fourier Transforms on Graphics Processors"
// (SC 2008): in a pass of radix R with span Ns, butterfly j reads
// x[j + r*N/R], applies the twiddles exp(-+2 pi i r (j mod Ns)/(Ns R)), runs an
// R-point DFT and writes y[(j/Ns)*Ns*R + j mod Ns + r*Ns].  N = E^s * R' with
// a final pass of radix R' < E in which each thread runs E/R' butterflies.
//
// Twiddles come from a host-computed table of exp(-2 pi i k / N) for the
// line length N (long double libm on the host, rounded once).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hos {


template <typename T>
struct CpxOf;
template <>
struct CpxOf<double> {
  using type = double2;
};
template <>
struct CpxOf<float> {
  using type = float2;
};
template <typename T>
using cpx = typename CpxOf<T>::type;

__device__ __forceinline__ double2 mkc(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mkc(float a, float b) { return make_float2(a, b); }

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  C r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  C r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a * conj(b)
template <typename C>
__device__ __forceinline__ C cmulc(C a, C b) {
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
template <typename C, typename S>
__device__ __forceinline__ C cscale(C a, S s) {
  C r;
  r.x = a.x * s;
  r.y = a.y * s;
  return r;
}
// multiply by i
template <typename C>
__device__ __forceinline__ C cmul_i(C a) {
  C r;
  r.x = -a.y;
  r.y = a.x;
  return r;
}
template <typename C>
__device__ __forceinline__ C cconj(C a) {
  C r;
  r.x = a.x;
  r.y = -a.y;
  return r;
}

__device__ __forceinline__ float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2((double)a.x, (double)a.y); }
template <typename T>
__device__ __forceinline__ cpx<T> conv(double2 a);
template <>
__device__ __forceinline__ double2 conv<double>(double2 a) {
  return a;
}
template <>
__device__ __forceinline__ float2 conv<float>(double2 a) {
  return to_f(a);
}
__device__ __forceinline__ double2 widen(double2 a) { return a; }
__device__ __forceinline__ double2 widen(float2 a) { return to_d(a); }

// cos(2 pi m / 32), m = 0..31, correctly rounded decimal literals.
__device__ __forceinline__ double cos32(int m) {
  switch (m & 31) {
    case 0: return 1.0;
    case 1: return 0.98078528040323044913;
    case 2: return 0.92387953251128675613;
    case 3: return 0.83146961230254523708;
    case 4: return 0.70710678118654752440;
    case 5: return 0.55557023301960222474;
    case 6: return 0.38268343236508977173;
    case 7: return 0.19509032201612826785;
    case 8: return 0.0;
    case 9: return -0.19509032201612826785;
    case 10: return -0.38268343236508977173;
    case 11: return -0.55557023301960222474;
    case 12: return -0.70710678118654752440;
    case 13: return -0.83146961230254523708;
    case 14: return -0.92387953251128675613;
    case 15: return -0.98078528040323044913;
    case 16: return -1.0;
    case 17: return -0.98078528040323044913;
    case 18: return -0.92387953251128675613;
    case 19: return -0.83146961230254523708;
    case 20: return -0.70710678118654752440;
    case 21: return -0.55557023301960222474;
    case 22: return -0.38268343236508977173;
    case 23: return -0.19509032201612826785;
    case 24: return 0.0;
    case 25: return 0.19509032201612826785;
    case 26: return 0.38268343236508977173;
    case 27: return 0.55557023301960222474;
    case 28: return 0.70710678118654752440;
    case 29: return 0.83146961230254523708;
    case 30: return 0.92387953251128675613;
    default: return 0.98078528040323044913;
  }
}

// b * exp(sgn * 2 pi i m / R) with R <= 32, m compile-time after unrolling.
template <int R, bool INV, typename C>
__device__ __forceinline__ C twc(C b, int m) {
  const int m32 = (m * (32 / R)) & 31;
  if (m32 == 0) return b;
  if (m32 == 8) {  // forward: times -i, inverse: times +i
    C r;
    r.x = INV ? -b.y : b.y;
    r.y = INV ? b.x : -b.x;
    return r;
  }
  if (m32 == 16) {
    C r;
    r.x = -b.x;
    r.y = -b.y;
    return r;
  }
  using S = decltype(b.x);
  S c = (S)cos32(m32);
  S s = (S)cos32(m32 - 8);  // sin(2 pi m32/32)
  if (!INV) s = -s;
  C w;
  w.x = c;
  w.y = s;
  return cmul(b, w);
}

// In-register R-point DFT (R in {2,4,8,16,32}), natural order in and out,
// forward exp(-i...), inverse exp(+i...), unnormalised.
template <int R>
__device__ __forceinline__ constexpr int bitrev(int i) {
  int r = 0;
  for (int b = 1, k = R >> 1; b < R; b <<= 1, k >>= 1)
    if (i & b) r |= k;
  return r;
}

template <int R, bool INV, typename C>
__device__ __forceinline__ void dft(C* a) {
  C b[R];
#pragma unroll
  for (int i = 0; i < R; i++) b[bitrev<R>(i)] = a[i];
#pragma unroll
  for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
    for (int i = 0; i < R; i += len) {
#pragma unroll
      for (int k = 0; k < len / 2; k++) {
        C u = b[i + k];
        C v = twc<R, INV>(b[i + k + len / 2], k * (R / len));
        b[i + k] = cadd(u, v);
        b[i + k + len / 2] = csub(u, v);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < R; i++) a[i] = b[i];
}

__host__ __device__ constexpr int hibit(int r) {
  int h = 1;
  while (h * 2 <= r) h *= 2;
  return h;
}

template <int N>
__device__ __forceinline__ constexpr int ilog2c() {
  int r = 0;
  for (int n = N; n > 1; n >>= 1) r++;
  return r;
}

// Shared-memory index of element a in the exchange after a pass of span ns.
// Elements are stored unpadded; within each 128-byte row (Q = 128 /
// sizeof(C) elements) the slot is XOR-swizzled so that both access patterns
// of the exchange are free of bank conflicts:
//   writes  a = (t/ns)*ns*E + t%ns + r*ns   (the radix-E butterfly outputs)
//   reads   a = t + e*P                      (consecutive threads)
// For ns >= Q the writes already come in runs of Q consecutive elements and
// no swizzle is needed.  Otherwise the bits of a that select the butterfly
// group (bits log2(ns*E)...) are folded into the slot bits above log2(ns).
template <int E, int Q>
__device__ __forceinline__ int sswz(int a, int ns) {
  if (ns >= Q) return a;
  const int mask = ((Q / ns) - 1) * ns;  // slot bits above log2(ns)
  return a ^ ((a >> ilog2c<E>()) & mask);
}
template <int N, int E>
__host__ __device__ constexpr int line_smem_elems() {
  return N;
}

// Twiddle exp(-+2 pi i a*scale / N) from the length-N table.
template <bool INV, typename C>
__device__ __forceinline__ C twid(const C* __restrict__ tw, int a, int scale) {
  C w = __ldg(&tw[a * scale]);
  if (INV) w.y = -w.y;
  return w;
}

// Barrier among the threads of one line.  A line of P <= 32 threads lies
// inside one warp (lines are consecutive thread ranges of power-of-two size),
// so a warp barrier suffices; larger lines use the block barrier, which every
// thread of the block reaches because all lines run the same passes.
template <int P>
__device__ __forceinline__ void line_sync() {
  if (P <= 32)
    __syncwarp();
  else
    __syncthreads();
}

template <int N, int E>
struct LinePlan {
  static constexpr int P = N / E;
  static constexpr int LOGE = ilog2c<E>();
  static constexpr int LOGN = ilog2c<N>();
  static constexpr int SFULL = LOGN / LOGE;  // full radix-E passes
  static constexpr int RLAST = 1 << (LOGN - SFULL * LOGE);
};

// Runs the line FFT in place on v.  All threads of the block must call it
// (it contains barriers); sm is this line's buffer of
// line_smem_elems<N,E>() elements; tw is the length-N twiddle table.
template <typename T, int N, int E, bool INV>
__device__ __forceinline__ void line_fft(cpx<T> (&v)[E], cpx<T>* sm, int t, const cpx<T>* __restrict__ tw) {
  using C = cpx<T>;
  using LP = LinePlan<N, E>;
  constexpr int P = LP::P;
  constexpr int SF = LP::SFULL;
  constexpr int RL = LP::RLAST;
  int ns = 1;
#pragma unroll
  for (int s = 0; s < SF; s++) {
    if (s > 0) {
      // twiddles w^r, w = exp(-+2 pi i jm/(ns E)): the powers w^(2^b) come
      // from the table and every other power is a product of those, so each
      // twiddle is at most log2(E)-1 products away from a table value
      const int jm = t & (ns - 1);
      const int scale = N / (ns * E);
      // w^r = w^(r - hi) * w^hi with hi the highest power of two in r: one
      // product per non-power r, at most log2(E)-1 products deep
      C wp[E];
#pragma unroll
      for (int b = 0; b < LP::LOGE; b++) wp[1 << b] = twid<INV>(tw, (1 << b) * jm, scale);
#pragma unroll
      for (int r = 3; r < E; r++) {
        const int hi = hibit(r);
        if (r != hi) wp[r] = cmul(wp[r - hi], wp[hi]);
      }
#pragma unroll
      for (int r = 1; r < E; r++) v[r] = cmul(v[r], wp[r]);
    }
    dft<E, INV>(v);
    const bool last = (s == SF - 1) && (RL == 1);
    if (!last) {
      constexpr int Q = 128 / (int)sizeof(C);
      line_sync<P>();
      // The swizzled slots are formed from one swizzled base per thread:
      // base has no bits where r*ns lies and the swizzle term never reads
      // those bits, so slot(base + r*ns) = slot(base) ^ r*ns; for the reads
      // (Q <= P) the term of e*P is a per-e constant below bit log2(P), so
      // slot(t + e*P) = (slot(t) ^ const_e) + e*P, an immediate offset.
      const int base = (t / ns) * ns * E + (t & (ns - 1));
      const int w0 = sswz<E, Q>(base, ns);
#pragma unroll
      for (int r = 0; r < E; r++) sm[w0 ^ (r * ns)] = v[r];
      line_sync<P>();
      if (Q <= P) {
        const int r0 = sswz<E, Q>(t, ns);
        const int mask = ns >= Q ? 0 : ((Q / ns) - 1) * ns;
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = sm[(r0 ^ (((e * P) >> LP::LOGE) & mask)) + e * P];
      } else {
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = sm[sswz<E, Q>(t + e * P, ns)];
      }
    }
    ns *= E;
  }
  if (RL > 1) {
    constexpr int Q = E / RL;
    const int scale = 1;
#pragma unroll
    for (int q = 0; q < Q; q++) {
      C a[RL > 1 ? RL : 1];
      const int j = t + q * P;
#pragma unroll
      for (int r = 0; r < RL; r++) {
        a[r] = v[q + r * Q];
        if (r > 0 && SF > 0) a[r] = cmul(a[r], twid<INV>(tw, r * j, scale));
      }
      dft<RL, INV>(a);
#pragma unroll
      for (int r = 0; r < RL; r++) v[q + r * Q] = a[r];
    }
  }
}

}  // namespace hos
