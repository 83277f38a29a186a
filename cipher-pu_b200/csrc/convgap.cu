// convgap.cu - coefficient-encoded RLWE inner products: the Conv + GAP
// fusion of an encrypted image, one ciphertext x plaintext product per filter.
//
//   ckks_mul_plain_multi: out[c][f] = (b_c w_f, a_c w_f) in Z_q[X]/(X^N + 1)
//     for every ciphertext c and weight polynomial f; the weights come in the
//     evaluation domain (forward negacyclic ckks_ntt, done once per model), so
//     each ciphertext polynomial costs one NTT and one INTT per filter.
//   ckks_decrypt_coef0: the constant coefficient of (b - a s) mod q, centred,
//     which is all an inner product reads of a decryption:
//     (a s)_0 = a_0 s_0 - sum_{i >= 1} a_i s_{N-i}.
#include "dispatch.cuh"
#include "profile.hpp"

// One CTA per (ciphertext, polynomial k); all global traffic lane-contiguous
// (layout C).  The transformed polynomial stays in registers across filters
// as exact doubles; each product is an FP64 modular multiply with w / q
// formed as w * (1 / q) (exact, within 1.5 q), fed to the inverse unreduced.
// Register budget: 512 resident threads per SM (128 registers a thread),
// 256 for K = 5 (255 registers).
template <int LOGN, int K>
struct MpmBlocks {
  static constexpr int T = NttShape<LOGN, K>::T;
  static constexpr int THR = K >= 5 ? 256 : 512;
  static constexpr int value = T >= THR ? 1 : (THR / T > 16 ? 16 : THR / T);
};

template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, (MpmBlocks<LOGN, K>::value))
    k_mul_plain_multi(u64* __restrict__ out, const u64* __restrict__ ct, const u64* __restrict__ w_hat,
                      int n_w, int prime, const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using S = NttShape<LOGN, K>;
  constexpr int N = S::N;
  const long long c = blockIdx.x >> 1;
  const int k = blockIdx.x & 1;
  const int tid = threadIdx.x;
  const PrimeInfo P = pi[prime];
  const TwD* tb = twbase<LOGN>(tw, prime);
  double x[S::E];
  {
    u64 xu[S::E];
    load_c<LOGN, K>(xu, ct + ((size_t)c * 2 + k) * N, tid);
#pragma unroll
    for (int e = 0; e < S::E; ++e) x[e] = u2d(reduce_any(xu[e], P));
  }
  ntt_fwd_d<LOGN, K>(x, sm, tid, tb, P);  // unreduced, |x| < 2^51
  if constexpr (S::NP == 0) __syncthreads();
  z_to_c<LOGN, K>(x, sm, tid);
#pragma unroll 1
  for (int f = 0; f < n_w; ++f) {
    double y[S::E];
#pragma unroll
    for (int e = 0; e < S::E; ++e) {
      const double w = u2d(reduce_any(w_hat[(size_t)f * N + posC<LOGN, K>(tid, e)], P));
      y[e] = fmulmod(x[e], w, __dmul_rn(w, P.qinv_d), P.qd);
    }
    __syncthreads();  // the previous filter's INTT is done with shared memory
    c_to_z<LOGN, K>(y, sm, tid);
    u64 yu[S::E];
    ntt_inv_d<LOGN, K>(y, yu, sm, tid, tb, P);
    store_c<LOGN, K>(yu, out + (((size_t)c * n_w + f) * 2 + k) * N, tid);
  }
}

// One warp per ciphertext.  Products are summed as exact 128-bit integers
// (residues below 2^52, at most N / 32 <= 512 terms a lane: below 2^113) and
// reduced once per lane.
__global__ void k_decrypt_coef0(long long* __restrict__ out, const u64* __restrict__ ct,
                                const u64* __restrict__ s, long long n_ct, int log_n, PrimeInfo P) {
  const long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= n_ct) return;  // uniform per warp
  const int n = 1 << log_n;
  const u64* b = ct + (size_t)c * 2 * n;
  const u64* a = b + n;
  u64 lo = 0, hi = 0;  // sum_{i >= 1} a_i s_{N-i}
#pragma unroll 8
  for (int i = lane ? lane : 32; i < n; i += 32) {
    const u64 av = ld_stream(a + i), sv = s[n - i];
    const u64 pl = av * sv;
    lo += pl;
    hi += __umul64hi(av, sv) + (lo < pl ? 1ull : 0ull);
  }
  u64 acc = addmod(reduce_any(lo, P), mulmod(reduce_any(hi, P), P.r_mod, P), P.q);
#pragma unroll
  for (int off = 16; off; off >>= 1) acc = addmod(acc, __shfl_down_sync(0xffffffffu, acc, off), P.q);
  if (lane == 0) {
    const u64 as0 = submod(mulmod(reduce_any(a[0], P), reduce_any(s[0], P), P), acc, P.q);
    const u64 d = submod(reduce_any(b[0], P), as0, P.q);
    out[c] = d > P.half ? (long long)d - (long long)P.q : (long long)d;
  }
}

extern "C" int ckks_mul_plain_multi(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct,
                                    const uint64_t* w_hat, int n_ct, int n_w, int prime, void* stream) {
  const char* fn = "ckks_mul_plain_multi";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(prime >= 0 && prime < ctx->n_primes, "%s: prime %d outside the %d context primes", fn, prime,
               ctx->n_primes);
  CKKS_REQUIRE(ctx->has_nega[prime], "%s: prime %d has no 2N-th root", fn, prime);
  CKKS_REQUIRE(n_ct >= 0 && n_w >= 0, "%s: negative count", fn);
  if (n_ct == 0 || n_w == 0) return CKKS_OK;
  CKKS_REQUIRE(out && ct && w_hat, "%s: NULL pointer argument", fn);
  cudaStream_t st = as_stream(stream);
  return dispatch_logn_k(ctx->log_n, ctx->tune_ntt_k, [&]<int L, int K>() -> int {
    using S = NttShape<L, K>;
    auto kern = k_mul_plain_multi<L, K>;
    if (int rc = require_smem(S::SMEM_WORDS * 8, L, fn)) return rc;
    ensure_smem(kern, S::SMEM_WORDS * 8);
    ProfSpan span(CKKS_STAGE_OTHER, st, "ckks conv + GAP: products per filter");
    kern<<<grid1d(2ll * n_ct), S::T, S::SMEM_WORDS * 8, st>>>(reinterpret_cast<u64*>(out),
                                                              reinterpret_cast<const u64*>(ct),
                                                              reinterpret_cast<const u64*>(w_hat), n_w,
                                                              prime, ctx->d_pi, ctx->d_tw);
    return ckks_check_launch(fn);
  }, fn);
}

extern "C" int ckks_decrypt_coef0(const ckks_ctx* ctx, int64_t* out, const uint64_t* ct, const uint64_t* s,
                                  long long n_ct, int prime, void* stream) {
  const char* fn = "ckks_decrypt_coef0";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(prime >= 0 && prime < ctx->n_primes, "%s: prime %d outside the %d context primes", fn, prime,
               ctx->n_primes);
  CKKS_REQUIRE(n_ct >= 0, "%s: n_ct < 0", fn);
  if (n_ct == 0) return CKKS_OK;
  CKKS_REQUIRE(out && ct && s, "%s: NULL pointer argument", fn);
  k_decrypt_coef0<<<grid1d((n_ct * 32 + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<long long*>(out), reinterpret_cast<const u64*>(ct), reinterpret_cast<const u64*>(s),
      n_ct, ctx->log_n, ctx->h_pi[prime]);
  return ckks_check_launch(fn);
}
