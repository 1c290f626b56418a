// x-pass kernel instantiations, double.
#include "hos_registry.h"

namespace hos {


template <int N, int E, int M, bool BT>
constexpr XInvFn xinv_fn() {
  if constexpr (elems_valid(0, N, E)) return &k_xinv<double, N, E, M, BT>;
  else return nullptr;
}
template <int N, int E, int M, bool BT>
constexpr XFwdFn xfwd_fn() {
  if constexpr (elems_valid(0, N, E)) return &k_xfwd<double, N, E, M, BT>;
  else return nullptr;
}

#define HOS_SIZES(F, E, M) F(16, E, M) F(32, E, M) F(64, E, M) F(128, E, M) F(256, E, M) F(512, E, M) \
  F(1024, E, M) F(2048, E, M) F(4096, E, M)

#define HOS_CASE_I(N, E, M) \
  case N:                   \
    return xinv_fn<N, E, M, BT>();
#define HOS_CASE_F(N, E, M) \
  case N:                   \
    return xfwd_fn<N, E, M, BT>();

template <int E, int M, bool BT>
static XInvFn xinv_n(int n) {
  switch (n) {
    HOS_SIZES(HOS_CASE_I, E, M)
    default: return nullptr;
  }
}
template <int E, int M, bool BT>
static XFwdFn xfwd_n(int n) {
  switch (n) {
    HOS_SIZES(HOS_CASE_F, E, M)
    default: return nullptr;
  }
}

template <int M, bool BT>
static XInvFn xinv_e(int n, int e) {
  switch (e) {
    case 8: return xinv_n<8, M, BT>(n);
    case 16: return xinv_n<16, M, BT>(n);
    case 32: return xinv_n<32, M, BT>(n);
    default: return nullptr;
  }
}
template <int M, bool BT>
static XFwdFn xfwd_e(int n, int e) {
  switch (e) {
    case 8: return xfwd_n<8, M, BT>(n);
    case 16: return xfwd_n<16, M, BT>(n);
    case 32: return xfwd_n<32, M, BT>(n);
    default: return nullptr;
  }
}

XInvFn lookup_xinv_64(int mode, int n, int e, bool batch) {
  switch (mode) {
    case XI_STAGE: return batch ? xinv_e<XI_STAGE, true>(n, e) : xinv_e<XI_STAGE, false>(n, e);
    case XI_PLAIN: return batch ? nullptr : xinv_e<XI_PLAIN, false>(n, e);
    default: return nullptr;
  }
}
XFwdFn lookup_xfwd_64(int mode, int n, int e, bool batch) {
  switch (mode) {
    case XF_PLAIN: return batch ? nullptr : xfwd_e<XF_PLAIN, false>(n, e);
    case XF_LEVEL: return batch ? xfwd_e<XF_LEVEL, true>(n, e) : xfwd_e<XF_LEVEL, false>(n, e);
    case XF_RHS: return batch ? xfwd_e<XF_RHS, true>(n, e) : xfwd_e<XF_RHS, false>(n, e);
    default: return nullptr;
  }
}

}  // namespace hos
