// x-pass kernel instantiations, double.
#include "hos_registry.h"

namespace hos {

#define HOS_X_CASE(N) \
  case N:             \
    return &k_xinv<double, N, elems_for(N)>;
XInvFn lookup_xinv_64(int n) {
  switch (n) {
    HOS_X_CASE(16) HOS_X_CASE(32) HOS_X_CASE(64) HOS_X_CASE(128) HOS_X_CASE(256) HOS_X_CASE(512)
    HOS_X_CASE(1024) HOS_X_CASE(2048) HOS_X_CASE(4096)
    default: return nullptr;
  }
}
#undef HOS_X_CASE
#define HOS_X_CASE(N) \
  case N:             \
    return &k_xfwd<double, N, elems_for(N)>;
XFwdFn lookup_xfwd_64(int n) {
  switch (n) {
    HOS_X_CASE(16) HOS_X_CASE(32) HOS_X_CASE(64) HOS_X_CASE(128) HOS_X_CASE(256) HOS_X_CASE(512)
    HOS_X_CASE(1024) HOS_X_CASE(2048) HOS_X_CASE(4096)
    default: return nullptr;
  }
}
#undef HOS_X_CASE

}  // namespace hos
