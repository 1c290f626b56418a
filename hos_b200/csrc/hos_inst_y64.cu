// y-pass kernel instantiations, double.
#include "hos_registry.h"

namespace hos {

#define HOS_Y_CASE(H) \
  case H:             \
    return &k_yinv<double, H, elems_for(H)>;
YInvFn lookup_yinv_64(int h) {
  switch (h) {
    HOS_Y_CASE(8) HOS_Y_CASE(16) HOS_Y_CASE(32) HOS_Y_CASE(64) HOS_Y_CASE(128) HOS_Y_CASE(256)
    HOS_Y_CASE(512) HOS_Y_CASE(1024) HOS_Y_CASE(2048)
    default: return nullptr;
  }
}
#undef HOS_Y_CASE
#define HOS_Y_CASE(H) \
  case H:             \
    return &k_yfwd<double, H, elems_for(H)>;
YFwdFn lookup_yfwd_64(int h) {
  switch (h) {
    HOS_Y_CASE(8) HOS_Y_CASE(16) HOS_Y_CASE(32) HOS_Y_CASE(64) HOS_Y_CASE(128) HOS_Y_CASE(256)
    HOS_Y_CASE(512) HOS_Y_CASE(1024) HOS_Y_CASE(2048)
    default: return nullptr;
  }
}
#undef HOS_Y_CASE

}  // namespace hos
