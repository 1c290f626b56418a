// x-pass kernel instantiations, double.
#include "hos_registry.h"

namespace hos {

#define HOS_SIZES(F) F(16) F(32) F(64) F(128) F(256) F(512) F(1024) F(2048) F(4096)

#define HOS_CASE(N) \
  case N:           \
    return &k_xinv<double, N, elems_for(N), M>;
template <int M>
static XInvFn xinv_n(int n) {
  switch (n) {
    HOS_SIZES(HOS_CASE)
    default: return nullptr;
  }
}
#undef HOS_CASE
#define HOS_CASE(N) \
  case N:           \
    return &k_xfwd<double, N, elems_for(N), M>;
template <int M>
static XFwdFn xfwd_n(int n) {
  switch (n) {
    HOS_SIZES(HOS_CASE)
    default: return nullptr;
  }
}
#undef HOS_CASE

XInvFn lookup_xinv_64(int mode, int n) {
  switch (mode) {
    case XI_STAGE: return xinv_n<XI_STAGE>(n);
    case XI_PLAIN: return xinv_n<XI_PLAIN>(n);
    default: return nullptr;
  }
}
XFwdFn lookup_xfwd_64(int mode, int n) {
  switch (mode) {
    case XF_PLAIN: return xfwd_n<XF_PLAIN>(n);
    case XF_LEVEL: return xfwd_n<XF_LEVEL>(n);
    case XF_RHS: return xfwd_n<XF_RHS>(n);
    default: return nullptr;
  }
}

}  // namespace hos
