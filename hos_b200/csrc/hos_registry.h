// Lookup of the compiled pass-kernel instantiations by precision, mode, line
// length and elements per thread.
#pragma once

#include "hos_kernels.cuh"

namespace hos {

using XInvFn = void (*)(XInvArgs, const XInvArgs*, const void*);
using XFwdFn = void (*)(XFwdArgs, const XFwdArgs*, const void*);
using YInvFn = void (*)(YInvArgs, const YInvArgs*, const void*, const void*);
using YFwdFn = void (*)(YFwdArgs, const YFwdArgs*, const void*, const void*);

// Elements per thread a line of length n is compiled for: 8 and 16 (n >= 16),
// and 32 in single precision (n >= 64); at most MAX_THREADS threads a line.
constexpr bool elems_valid(int prec, int n, int e) {
  return (e == 8 || e == 16 || (e == 32 && prec == 1)) && n >= e && n / e <= MAX_THREADS && (e != 32 || n >= 64);
}

// prec: 0 = double, 1 = float; batch: per-field arguments from a device
// array indexed by blockIdx.z.  Return nullptr for an unsupported combination.
XInvFn lookup_xinv(int prec, int mode, int n, int e, bool batch = false);
XFwdFn lookup_xfwd(int prec, int mode, int n, int e, bool batch = false);
YInvFn lookup_yinv(int prec, int mode, int h, int e, bool batch = false);
YFwdFn lookup_yfwd(int prec, int mode, int h, int e, bool batch = false);

}  // namespace hos
