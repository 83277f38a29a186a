// rescale.cu - the golden single-modulus rescales (exact and scaled) and the
// RNS drop-last-limb rescale.
#include "dispatch.cuh"
#include "profile.hpp"

// round(c * q_out / q_in) mod q_out, round half up (scripts/verify_rescale.py:38).
__global__ void k_rescale_exact(u64* __restrict__ out, const u64* __restrict__ in, long long n,
                                u64 q_in, u64 q_out, double ratio) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const u64 c = in[idx];
  // quotient estimate of floor(c * q_out / q_in); |error| <= 1
  u64 r = (u64)floor(__dmul_rn(__ull2double_rn(c), ratio));
  i64 rem = (i64)(c * q_out - r * q_in);  // exact: |rem| < 2^52
  if (rem < 0) { rem += (i64)q_in; --r; }
  if (rem < 0) { rem += (i64)q_in; --r; }
  if (rem >= (i64)q_in) { rem -= (i64)q_in; ++r; }
  if (rem >= (i64)q_in) { rem -= (i64)q_in; ++r; }
  if (2 * (u64)rem >= q_in) ++r;
  out[idx] = r % q_out;
}

extern "C" int ckks_rescale_exact(uint64_t* out, const uint64_t* in, int64_t n, uint64_t q_in,
                                  uint64_t q_out, void* stream) {
  CKKS_REQUIRE(n >= 0, "ckks_rescale_exact: n < 0");
  CKKS_REQUIRE(q_in >= 2 && q_in < (1ull << 50) && q_out >= 1 && q_out < (1ull << 50),
               "ckks_rescale_exact: moduli must lie in [2, 2^50)");
  if (n == 0) return CKKS_OK;
  k_rescale_exact<<<grid1d((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), n, q_in, q_out,
      (double)q_out / (double)q_in);
  return ckks_check_launch("ckks_rescale_exact");
}

// floor((s * q_out + q_in / 2) / (q_in * 2^sb)) mod q_out (scripts/verify_e2e_mult.py:70).
// floor(x / (q_in 2^sb)) = floor(floor(x / 2^sb) / q_in).
__global__ void k_rescale_scaled(u64* __restrict__ out, const u64* __restrict__ in, long long n,
                                 u64 q_in, u64 q_out, int sb) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const u64 s = in[idx];
  u64 lo = s * q_out;
  u64 hi = __umul64hi(s, q_out);
  const u64 add = q_in / 2;
  const u64 lo2 = lo + add;
  hi += (lo2 < lo) ? 1 : 0;
  lo = lo2;
  if (sb > 0) {  // 128-bit logical shift right by sb (sb < 64)
    lo = (lo >> sb) | (hi << (64 - sb));
    hi >>= sb;
  }
  // x = hi:lo, floor(x / q_in); x < 2^100 so a double estimate is within +-1 of the
  // quotient when the quotient is < 2^53; the remainder is exact in the low word.
  const double xd = __dadd_rn(__dmul_rn(__ull2double_rn(hi), 18446744073709551616.0),
                              __ull2double_rn(lo));
  u64 r = (u64)floor(xd / (double)q_in);
  i64 rem = (i64)(lo - r * q_in);
  for (int it = 0; it < 4 && rem < 0; ++it) { rem += (i64)q_in; --r; }
  for (int it = 0; it < 4 && rem >= (i64)q_in; ++it) { rem -= (i64)q_in; ++r; }
  out[idx] = r % q_out;
}

extern "C" int ckks_rescale_scaled(uint64_t* out, const uint64_t* in, int64_t n, uint64_t q_in,
                                   uint64_t q_out, int scale_bits, void* stream) {
  CKKS_REQUIRE(n >= 0, "ckks_rescale_scaled: n < 0");
  CKKS_REQUIRE(q_in >= 2 && q_in < (1ull << 50) && q_out >= 1 && q_out < (1ull << 50),
               "ckks_rescale_scaled: moduli must lie in [2, 2^50)");
  CKKS_REQUIRE(scale_bits >= 0 && scale_bits < 64, "ckks_rescale_scaled: scale_bits outside [0, 64)");
  if (n == 0) return CKKS_OK;
  k_rescale_scaled<<<grid1d((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), n, q_in, q_out, scale_bits);
  return ckks_check_launch("ckks_rescale_scaled");
}

// ------------------------------------------------------------------ RNS rescale
// One CTA per polynomial: INTT the last limb, centre it, and for every
// remaining limb i: out_i = (x_i - NTT_i([w]_{q_i})) * q_t^-1.
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_rescale_rns(u64* __restrict__ out, const u64* __restrict__ in, int level,
                  const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw,
                  const TwPair* __restrict__ qtinv, int nq) {
  extern __shared__ u64 sm[];
  using S = NttShape<LOGN, K>;
  const long long poly = blockIdx.x;
  const int t = level - 1;
  const int tid = threadIdx.x;
  const u64* src = in + (size_t)poly * level * S::N;
  u64* dst = out + (size_t)poly * t * S::N;
  const PrimeInfo PT = pi[t];
  u64 w[S::E];
  load_c<LOGN, K>(w, src + (size_t)t * S::N, tid);
  c_to_z<LOGN, K>(w, sm, tid);
  ntt_inv<LOGN, K>(w, sm, tid, twbase<LOGN>(tw, t), PT);
#pragma unroll 1
  for (int i = 0; i < t; ++i) {
    const PrimeInfo P = pi[i];
    const TwPair ci = qtinv[(size_t)t * nq + i];
    u64 x[S::E];
#pragma unroll
    for (int e = 0; e < S::E; ++e) x[e] = w[e] > PT.half ? w[e] - PT.q + P.q : w[e];  // [w_c]_{q_i}
    ntt_fwd<LOGN, K>(x, sm, tid, twbase<LOGN>(tw, i), P);
    z_to_c<LOGN, K>(x, sm, tid);
    u64 xi[S::E];
    load_c<LOGN, K>(xi, src + (size_t)i * S::N, tid);
#pragma unroll
    for (int e = 0; e < S::E; ++e) x[e] = shoup(xi[e] + P.qlazy - x[e], ci.w, ci.ws, P.q);
    store_c<LOGN, K>(x, dst + (size_t)i * S::N, tid);
  }
}

extern "C" int ckks_rescale_rns(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in,
                                int n_polys, int level, void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks RNS rescale");
  CKKS_REQUIRE(ctx != nullptr, "ckks_rescale_rns: ctx is NULL");
  CKKS_REQUIRE(level >= 2 && level <= ctx->n_q, "ckks_rescale_rns: level=%d outside [2, %d]",
               level, ctx->n_q);
  CKKS_REQUIRE(out != in, "ckks_rescale_rns: out must differ from in");
  for (int i = 0; i < level; ++i)
    CKKS_REQUIRE(ctx->has_nega[i], "ckks_rescale_rns: prime %d has no 2N-th root", i);
  for (int i = 0; i < level - 1; ++i)
    CKKS_REQUIRE(ctx->primes[level - 1] < 2 * ctx->primes[i],
                 "ckks_rescale_rns: q_%d must be < 2 q_%d for the centred conversion", level - 1, i);
  if (n_polys <= 0) return CKKS_OK;
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    using S = NttShape<L, K>;
    auto kern = k_rescale_rns<L, K>;
    ensure_smem(kern, S::SMEM_WORDS * 8);
    kern<<<grid1d(n_polys), S::T, S::SMEM_WORDS * 8, as_stream(stream)>>>(
        reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), level, ctx->d_pi,
        ctx->d_tw, ctx->d_qtinv, ctx->n_q);
    return ckks_check_launch("ckks_rescale_rns");
  });
}
