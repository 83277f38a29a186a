// dispatch.cuh - compile-time dispatch over the ring dimension and launch
// helpers shared by the kernel files.
#pragma once
#include "ctx.hpp"
#include "ntt.cuh"

// K (log2 coefficients per thread) used for a given log N.
template <int LOGN>
struct DefaultK {
  static constexpr int value = LOGN < 4 ? LOGN : 4;
};

// Calls F.template operator()<LOGN, K>() for the runtime log_n.
template <typename F>
static int dispatch_logn(int log_n, F&& f) {
  switch (log_n) {
#define CKKS_CASE(L) \
  case L:            \
    return f.template operator()<L, DefaultK<L>::value>();
    CKKS_CASE(1)
    CKKS_CASE(2)
    CKKS_CASE(3)
    CKKS_CASE(4)
    CKKS_CASE(5)
    CKKS_CASE(6)
    CKKS_CASE(7)
    CKKS_CASE(8)
    CKKS_CASE(9)
    CKKS_CASE(10)
    CKKS_CASE(11)
    CKKS_CASE(12)
    CKKS_CASE(13)
    CKKS_CASE(14)
#undef CKKS_CASE
    default:
      return ckks_set_error(CKKS_EUNSUPPORTED, "log_n=%d unsupported", log_n);
  }
}

// dispatch_logn with a tuned K: k = 0 takes DefaultK, k in [2, 5] is built
// for log N in [6, 14] with N / 2^K <= 1024 threads.
template <typename F>
static int dispatch_logn_k(int log_n, int k, F&& f, const char* fn) {
  if (k == 0) return dispatch_logn(log_n, f);
  if (k < 2 || k > 5 || log_n < 6 || log_n > 14 || ((1 << log_n) >> k) > 1024)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: K=%d not built at log_n=%d", fn, k, log_n);
  auto go = [&]<int L>() -> int {
    switch (k) {
      case 2:
        if constexpr (((1 << L) >> 2) <= 1024) return f.template operator()<L, 2>();
        break;
      case 3:
        if constexpr (((1 << L) >> 3) <= 1024) return f.template operator()<L, 3>();
        break;
      case 4:
        return f.template operator()<L, 4>();
      default:
        return f.template operator()<L, 5>();
    }
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: K=%d not built at log_n=%d", fn, k, log_n);
  };
  switch (log_n) {
    case 6: return go.template operator()<6>();
    case 7: return go.template operator()<7>();
    case 8: return go.template operator()<8>();
    case 9: return go.template operator()<9>();
    case 10: return go.template operator()<10>();
    case 11: return go.template operator()<11>();
    case 12: return go.template operator()<12>();
    case 13: return go.template operator()<13>();
    default: return go.template operator()<14>();
  }
}

// Opt a kernel into > 48 KB of dynamic shared memory once per process/device.
template <typename KernelT>
static cudaError_t ensure_smem(KernelT kernel, int bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

static inline unsigned grid1d(long long blocks) { return (unsigned)blocks; }

// Largest dynamic shared memory a CTA may opt into on the current device.
static inline int smem_optin_limit() {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return v;
}

// Error unless `bytes` of dynamic shared memory per CTA fit on this device.
static inline int require_smem(int bytes, int log_n, const char* fn) {
  const int lim = smem_optin_limit();
  if (bytes > lim)
    return ckks_set_error(CKKS_EUNSUPPORTED,
                          "%s: N=2^%d needs %d KB of shared memory per CTA, above the device's %d KB",
                          fn, log_n, bytes / 1024, lim / 1024);
  return CKKS_OK;
}
