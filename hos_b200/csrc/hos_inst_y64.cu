// y-pass kernel instantiations, double.
#include "hos_registry.h"

namespace hos {

template <int H, int E, int M>
constexpr YInvFn yinv_fn() {
  if constexpr (elems_valid(0, H, E)) return &k_yinv<double, H, E, M>;
  else return nullptr;
}
template <int H, int E, int M>
constexpr YFwdFn yfwd_fn() {
  if constexpr (elems_valid(0, H, E)) return &k_yfwd<double, H, E, M>;
  else return nullptr;
}

#define HOS_SIZES(F, E, M) F(8, E, M) F(16, E, M) F(32, E, M) F(64, E, M) F(128, E, M) F(256, E, M) F(512, E, M) \
  F(1024, E, M) F(2048, E, M)

#define HOS_CASE_I(H, E, M) \
  case H:                   \
    return yinv_fn<H, E, M>();
#define HOS_CASE_F(H, E, M) \
  case H:                   \
    return yfwd_fn<H, E, M>();

template <int E, int M>
static YInvFn yinv_n(int h) {
  switch (h) {
    HOS_SIZES(HOS_CASE_I, E, M)
    default: return nullptr;
  }
}
template <int E, int M>
static YFwdFn yfwd_n(int h) {
  switch (h) {
    HOS_SIZES(HOS_CASE_F, E, M)
    default: return nullptr;
  }
}
template <int M>
static YInvFn yinv_e(int h, int e) {
  switch (e) {
    case 8: return yinv_n<8, M>(h);
    case 16: return yinv_n<16, M>(h);
    case 32: return yinv_n<32, M>(h);
    default: return nullptr;
  }
}
template <int M>
static YFwdFn yfwd_e(int h, int e) {
  switch (e) {
    case 8: return yfwd_n<8, M>(h);
    case 16: return yfwd_n<16, M>(h);
    case 32: return yfwd_n<32, M>(h);
    default: return nullptr;
  }
}

YInvFn lookup_yinv_64(int mode, int h, int e) {
  switch (mode) {
    case YI_JOBS: return yinv_e<YI_JOBS>(h, e);
    case YI_LEVEL: return yinv_e<YI_LEVEL>(h, e);
    default: return nullptr;
  }
}
YFwdFn lookup_yfwd_64(int mode, int h, int e) {
  switch (mode) {
    case YF_PLAIN: return yfwd_e<YF_PLAIN>(h, e);
    case YF_LEVEL: return yfwd_e<YF_LEVEL>(h, e);
    case YF_RHS: return yfwd_e<YF_RHS>(h, e);
    default: return nullptr;
  }
}

}  // namespace hos
