// Lookup of the compiled pass-kernel instantiations by precision, mode and
// line length.
#pragma once

#include "hos_kernels.cuh"

namespace hos {

using XInvFn = void (*)(XInvArgs, const void*);
using XFwdFn = void (*)(XFwdArgs, const void*);
using YInvFn = void (*)(YInvArgs, const void*, const void*);
using YFwdFn = void (*)(YFwdArgs, const void*, const void*);

// Elements per thread chosen for a line length (one instantiation per length).
constexpr int elems_for(int n) { return n <= 8 ? n : (n <= 2048 ? 8 : 16); }

// prec: 0 = double, 1 = float.  Return nullptr for an unsupported length.
XInvFn lookup_xinv(int prec, int mode, int n);
XFwdFn lookup_xfwd(int prec, int mode, int n);
YInvFn lookup_yinv(int prec, int mode, int h);
YFwdFn lookup_yfwd(int prec, int mode, int h);

}  // namespace hos
