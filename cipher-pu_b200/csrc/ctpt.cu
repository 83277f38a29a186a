// ctpt.cu - ciphertext x plaintext multiply fused with the RNS rescale.
//
// One CTA per (ct, poly k) (body: ctpt_unit, ctmul_units.cuh).  The
// plaintext may be shared by all ciphertexts (pt_stride = 0) or given per
// ciphertext (pt_stride = 1).
#include "ctmul_units.cuh"
#include "dispatch.cuh"
#include "profile.hpp"

// Register budget: resident threads per SM targeted per K (128 registers a
// thread at K = 4, 64 at K <= 3, ~240 for the 32 values a thread of K = 5).
template <int LOGN, int K>
struct CtptBlocks {
  static constexpr int T = NttShape<LOGN, K>::T;
  static constexpr int THR = K >= 5 ? 256 : (K == 4 ? 512 : 1024);
  static constexpr int value = T >= THR ? 1 : THR / T;
};

template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, (CtptBlocks<LOGN, K>::value))
    k_ctpt_rescale(u64* __restrict__ out, const u64* __restrict__ ct, const u64* __restrict__ pt,
                   int pt_stride, int level, const PrimeInfo* __restrict__ pi,
                   const TwD* __restrict__ tw, const TwPair* __restrict__ qtinv, int nq) {
  extern __shared__ u64 sm[];
  ctpt_unit<LOGN, K>(out, ct, pt, pt_stride, level, pi, tw, qtinv, nq, blockIdx.x >> 1, blockIdx.x & 1, sm,
                     threadIdx.x);
}

extern "C" int ckks_ct_mul_plain_rescale(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct,
                                         const uint64_t* pt, int pt_per_ct, int n_ct, int level,
                                         void* stream) {
  const char* fn = "ckks_ct_mul_plain_rescale";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(level >= 2 && level <= ctx->n_q, "%s: level=%d outside [2, %d]", fn, level, ctx->n_q);
  CKKS_REQUIRE(n_ct >= 0, "%s: n_ct < 0", fn);
  for (int i = 0; i < level; ++i)
    CKKS_REQUIRE(ctx->has_nega[i], "%s: prime %d has no 2N-th root", fn, i);
  for (int i = 0; i < level - 1; ++i)
    CKKS_REQUIRE(ctx->primes[level - 1] < 2 * ctx->primes[i],
                 "%s: q_%d must be < 2 q_%d for the centred conversion", fn, level - 1, i);
  if (n_ct == 0) return CKKS_OK;
  CKKS_REQUIRE(out && ct && pt, "%s: NULL pointer argument", fn);
  cudaStream_t st = as_stream(stream);
  return dispatch_logn_k(ctx->log_n, ctx->tune_ntt_k, [&]<int L, int K>() -> int {
    using Sh = NttShape<L, K>;
    const int smem = (Sh::SMEM_WORDS + Sh::N) * 8;
    if (int rc = require_smem(smem, L, fn)) return rc;
    ensure_smem(k_ctpt_rescale<L, K>, smem);
    ProfSpan span(CKKS_STAGE_OTHER, st, "ckks ct x pt + rescale");
    k_ctpt_rescale<L, K><<<grid1d(2ll * n_ct), Sh::T, smem, st>>>(
        reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(ct), reinterpret_cast<const u64*>(pt),
        pt_per_ct ? 1 : 0, level, ctx->d_pi, ctx->d_tw, ctx->d_qtinv, ctx->n_q);
    return ckks_check_launch(fn);
  }, fn);
}
