// y-pass kernel instantiations, float.
#include "hos_registry.h"

namespace hos {

#define HOS_SIZES(F) F(8) F(16) F(32) F(64) F(128) F(256) F(512) F(1024) F(2048)

#define HOS_CASE(H) \
  case H:           \
    return &k_yinv<float, H, elems_for(H), M>;
template <int M>
static YInvFn yinv_h(int h) {
  switch (h) {
    HOS_SIZES(HOS_CASE)
    default: return nullptr;
  }
}
#undef HOS_CASE
#define HOS_CASE(H) \
  case H:           \
    return &k_yfwd<float, H, elems_for(H), M>;
template <int M>
static YFwdFn yfwd_h(int h) {
  switch (h) {
    HOS_SIZES(HOS_CASE)
    default: return nullptr;
  }
}
#undef HOS_CASE

YInvFn lookup_yinv_32(int mode, int h) {
  switch (mode) {
    case YI_JOBS: return yinv_h<YI_JOBS>(h);
    case YI_LEVEL: return yinv_h<YI_LEVEL>(h);
    default: return nullptr;
  }
}
YFwdFn lookup_yfwd_32(int mode, int h) {
  switch (mode) {
    case YF_PLAIN: return yfwd_h<YF_PLAIN>(h);
    case YF_LEVEL: return yfwd_h<YF_LEVEL>(h);
    case YF_RHS: return yfwd_h<YF_RHS>(h);
    default: return nullptr;
  }
}

}  // namespace hos
