// peak.cu - modular-multiply throughput microbenchmark (the compute roofline
// of the NTT-bound kernels): every thread runs 8 independent chains of
// lazy modular multiplies by a fixed twiddle, with 45-bit primes.
//   kind 0: integer Shoup (mul.hi.u64 quotient, two low products) - the
//           arithmetic of the butterflies;
//   kind 1: FP64 double-word product (exact a*w = hi + lo via FMA, quotient by
//           a rounding FMA against 1.5 * 2^52, exact remainder by FMA);
//   kind 2: half the chains of each kind, interleaved.
#include "dispatch.cuh"

constexpr int PK_CHAINS = 8;

__global__ void k_peak(u64* __restrict__ out, int iters, int kind, u64 q, u64 w, u64 ws, double qd,
                       double wd, double wqd) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  u64 xi[PK_CHAINS];
  double xd[PK_CHAINS];
#pragma unroll
  for (int c = 0; c < PK_CHAINS; ++c) {
    xi[c] = (u64)(tid * 7919 + c * 104729) % q;
    xd[c] = (double)xi[c];
  }
  const double magic = 6755399441055744.0;  // 1.5 * 2^52
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) {
      const bool use_fp = kind == 1 || (kind == 2 && (c & 1));
      if (!use_fp) {
        xi[c] = shoup_lazy(xi[c], w, ws, q);
      } else {
        const double hi = xd[c] * wd;
        const double lo = fma(xd[c], wd, -hi);
        const double qt = fma(xd[c], wqd, magic) - magic;
        double r = fma(-qt, qd, hi) + lo;   // exact, in (-q, 2q)
        r = r < 0.0 ? r + qd : r;
        xd[c] = r;
      }
    }
  }
  u64 acc = 0;
#pragma unroll
  for (int c = 0; c < PK_CHAINS; ++c) acc += xi[c] + (u64)xd[c];
  out[tid] = acc;
}

extern "C" int ckks_modmul_peak(uint64_t* out, int n_blocks, int threads, int iters, int kind,
                                uint64_t q, uint64_t w, void* stream) {
  CKKS_REQUIRE(out && n_blocks > 0 && threads > 0 && threads <= 1024 && iters > 0,
               "ckks_modmul_peak: bad launch shape");
  CKKS_REQUIRE(kind >= 0 && kind <= 2, "ckks_modmul_peak: kind outside [0, 2]");
  CKKS_REQUIRE(q > 2 && q < (1ull << 47) && w < q, "ckks_modmul_peak: need w < q < 2^47");
  const u64 ws = h_shoup(w, q);
  k_peak<<<n_blocks, threads, 0, as_stream(stream)>>>(reinterpret_cast<u64*>(out), iters, kind, q, w,
                                                      ws, (double)q, (double)w,
                                                      (double)w / (double)q);
  return ckks_check_launch("ckks_modmul_peak");
}
