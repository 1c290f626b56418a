// y-pass kernel instantiations, float.
#include "hos_registry.h"

namespace hos {

template <int H, int E, int M, bool BT>
constexpr YInvFn yinv_fn() {
  if constexpr (elems_valid(1, H, E)) return &k_yinv<float, H, E, M, BT>;
  else return nullptr;
}
template <int H, int E, int M, bool BT>
constexpr YFwdFn yfwd_fn() {
  if constexpr (elems_valid(1, H, E)) return &k_yfwd<float, H, E, M, BT>;
  else return nullptr;
}

#define HOS_SIZES(F, E, M) F(8, E, M) F(16, E, M) F(32, E, M) F(64, E, M) F(128, E, M) F(256, E, M) F(512, E, M) \
  F(1024, E, M) F(2048, E, M)

#define HOS_CASE_I(H, E, M) \
  case H:                   \
    return yinv_fn<H, E, M, BT>();
#define HOS_CASE_F(H, E, M) \
  case H:                   \
    return yfwd_fn<H, E, M, BT>();

template <int E, int M, bool BT>
static YInvFn yinv_n(int h) {
  switch (h) {
    HOS_SIZES(HOS_CASE_I, E, M)
    default: return nullptr;
  }
}
template <int E, int M, bool BT>
static YFwdFn yfwd_n(int h) {
  switch (h) {
    HOS_SIZES(HOS_CASE_F, E, M)
    default: return nullptr;
  }
}
template <int M, bool BT>
static YInvFn yinv_e(int h, int e) {
  switch (e) {
    case 8: return yinv_n<8, M, BT>(h);
    case 16: return yinv_n<16, M, BT>(h);
    case 32: return yinv_n<32, M, BT>(h);
    default: return nullptr;
  }
}
template <int M, bool BT>
static YFwdFn yfwd_e(int h, int e) {
  switch (e) {
    case 8: return yfwd_n<8, M, BT>(h);
    case 16: return yfwd_n<16, M, BT>(h);
    case 32: return yfwd_n<32, M, BT>(h);
    default: return nullptr;
  }
}

YInvFn lookup_yinv_32(int mode, int h, int e, bool batch) {
  switch (mode) {
    case YI_JOBS: return batch ? yinv_e<YI_JOBS, true>(h, e) : yinv_e<YI_JOBS, false>(h, e);
    case YI_LEVEL: return batch ? yinv_e<YI_LEVEL, true>(h, e) : yinv_e<YI_LEVEL, false>(h, e);
    default: return nullptr;
  }
}
YFwdFn lookup_yfwd_32(int mode, int h, int e, bool batch) {
  switch (mode) {
    case YF_PLAIN: return batch ? nullptr : yfwd_e<YF_PLAIN, false>(h, e);
    case YF_LEVEL: return batch ? yfwd_e<YF_LEVEL, true>(h, e) : yfwd_e<YF_LEVEL, false>(h, e);
    case YF_RHS: return batch ? yfwd_e<YF_RHS, true>(h, e) : yfwd_e<YF_RHS, false>(h, e);
    default: return nullptr;
  }
}

}  // namespace hos
