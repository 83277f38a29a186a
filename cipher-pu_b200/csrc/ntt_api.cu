// ntt_api.cu - batched NTT, permutation, pointwise and fused polynomial
// product kernels behind the C ABI (golden-model path and building blocks).
#include "dispatch.cuh"
#include "profile.hpp"

// ------------------------------------------------------------------ NTT
// One CTA per limb-transform.  Limb-major grid (blockIdx = limb * n_polys +
// poly), so the CTAs resident on an SM at a time share one prime's twiddle
// tables in L1.  Global traffic is lane-contiguous (layout C) both ways; the
// forward's layout-Z result is re-distributed through shared memory first.
// CTAs per SM the standalone transform's register budget targets: three
// 256-thread CTAs (85 registers) where the CTA is small enough; for K = 5
// (32 values per thread) 256 resident threads (255 registers).
template <int LOGN, int K>
struct NttMinBlocks {
  static constexpr int T = NttShape<LOGN, K>::T;
  static constexpr int THR = K >= 5 ? 256 : 768;
  static constexpr int value = T >= THR ? 1 : (THR / T > 8 ? 8 : THR / T);
};

template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, (NttMinBlocks<LOGN, K>::value))
    k_ntt(u64* __restrict__ data, int n_polys, int n_limbs, int prime_begin,
          const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw, int inverse, int cyclic) {
  extern __shared__ u64 sm[];
  using S = NttShape<LOGN, K>;
  const int limb = blockIdx.x / n_polys;
  const long long poly = blockIdx.x % n_polys;
  const int pidx = prime_begin + limb;
  const PrimeInfo P = pi[pidx];
  u64* d = data + ((size_t)poly * n_limbs + limb) * S::N;
  const TwD* tb = twbase<LOGN>(tw, pidx);
  const int tid = threadIdx.x;
  u64 x[S::E];
#pragma unroll
  for (int e = 0; e < S::E; ++e) x[e] = reduce_any(ld_stream(d + posC<LOGN, K>(tid, e)), P);
  if (!inverse) {
    ntt_fwd<LOGN, K>(x, sm, tid, tb, P, cyclic);
    if constexpr (S::NP == 0) __syncthreads();
    z_to_c<LOGN, K>(x, sm, tid);
  } else {
    c_to_z<LOGN, K>(x, sm, tid);
    ntt_inv<LOGN, K>(x, sm, tid, tb, P, cyclic);
  }
  store_c<LOGN, K>(x, d, tid);
}

static int check_limbs(const ckks_ctx* ctx, int prime_begin, int n_limbs, const char* fn) {
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_limbs >= 1 && prime_begin >= 0 && prime_begin + n_limbs <= ctx->n_primes,
               "%s: limb range [%d, %d) outside the %d context primes", fn, prime_begin,
               prime_begin + n_limbs, ctx->n_primes);
  return CKKS_OK;
}

extern "C" int ckks_ntt(const ckks_ctx* ctx, uint64_t* data, int n_polys, int prime_begin,
                        int n_limbs, int inverse, int cyclic, void* stream) {
  if (int rc = check_limbs(ctx, prime_begin, n_limbs, "ckks_ntt")) return rc;
  CKKS_REQUIRE(n_polys >= 0, "ckks_ntt: n_polys < 0");
  if (!cyclic)
    for (int l = 0; l < n_limbs; ++l)
      CKKS_REQUIRE(ctx->has_nega[prime_begin + l],
                   "ckks_ntt: prime %d has no 2N-th root; negacyclic transform unavailable",
                   prime_begin + l);
  if (n_polys == 0) return CKKS_OK;
  CKKS_REQUIRE(data != nullptr, "ckks_ntt: data is NULL");
  auto launch = [&]<int L, int K>() -> int {
    using S = NttShape<L, K>;
    auto kern = k_ntt<L, K>;
    ensure_smem(kern, S::SMEM_WORDS * 8);
    ProfSpan span(CKKS_STAGE_NTT, as_stream(stream));
    kern<<<grid1d((long long)n_polys * n_limbs), S::T, S::SMEM_WORDS * 8, as_stream(stream)>>>(
        reinterpret_cast<u64*>(data), n_polys, n_limbs, prime_begin, ctx->d_pi, ctx->d_tw, inverse,
        cyclic);
    return ckks_check_launch("ckks_ntt");
  };
  return dispatch_logn_k(ctx->log_n, ctx->tune_ntt_k, launch, "ckks_ntt");
}

// ------------------------------------------------------------------ bitrev
__global__ void k_bitrev(u64* __restrict__ out, const u64* __restrict__ in, long long total,
                         int log_n) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const long long row = idx >> log_n;
  const unsigned i = (unsigned)(idx & ((1ll << log_n) - 1));
  const unsigned j = __brev(i) >> (32 - log_n);
  out[idx] = in[(row << log_n) + j];
}

extern "C" int ckks_bitrev_permute(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in,
                                   int n_rows, void* stream) {
  CKKS_REQUIRE(ctx != nullptr, "ckks_bitrev_permute: ctx is NULL");
  CKKS_REQUIRE(n_rows >= 0, "ckks_bitrev_permute: n_rows < 0");
  CKKS_REQUIRE(out != in, "ckks_bitrev_permute: out must differ from in");
  const long long total = (long long)n_rows << ctx->log_n;
  if (total == 0) return CKKS_OK;
  k_bitrev<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), total, ctx->log_n);
  return ckks_check_launch("ckks_bitrev_permute");
}

// ------------------------------------------------------------------ pointwise
__global__ void k_pointwise(u64* __restrict__ out, const u64* __restrict__ a,
                            const u64* __restrict__ b, long long total, int log_n, int n_limbs,
                            int prime_begin, const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int limb = (int)((idx >> log_n) % n_limbs);
  const PrimeInfo P = pi[prime_begin + limb];
  out[idx] = mulmod(a[idx], b[idx], P);
}

extern "C" int ckks_pointwise_mul(const ckks_ctx* ctx, uint64_t* out, const uint64_t* a,
                                  const uint64_t* b, int n_polys, int prime_begin, int n_limbs,
                                  void* stream) {
  if (int rc = check_limbs(ctx, prime_begin, n_limbs, "ckks_pointwise_mul")) return rc;
  const long long total = ((long long)n_polys * n_limbs) << ctx->log_n;
  if (total <= 0) return CKKS_OK;
  k_pointwise<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(a),
      reinterpret_cast<const u64*>(b), total, ctx->log_n, n_limbs, prime_begin, ctx->d_pi);
  return ckks_check_launch("ckks_pointwise_mul");
}

// ------------------------------------------------------------------ add / sub
__global__ void k_addsub(u64* __restrict__ out, const u64* __restrict__ a,
                         const u64* __restrict__ b, long long n, u64 q, int subtract) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const u64 x = a[idx], y = b[idx];
  out[idx] = subtract ? submod(x, y, q) : addmod(x, y, q);
}

extern "C" int ckks_vec_addsub(uint64_t* out, const uint64_t* a, const uint64_t* b, int64_t n,
                               uint64_t q, int subtract, void* stream) {
  CKKS_REQUIRE(n >= 0, "ckks_vec_addsub: n < 0");
  CKKS_REQUIRE(q >= 2 && q < (1ull << 62), "ckks_vec_addsub: q outside [2, 2^62)");
  if (n == 0) return CKKS_OK;
  k_addsub<<<grid1d((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(a),
      reinterpret_cast<const u64*>(b), n, q, subtract);
  return ckks_check_launch("ckks_vec_addsub");
}

// ------------------------------------------------------------------ poly mul
// One CTA per polynomial limb: both operands transformed (unreduced FP64),
// reduced to |x| <= q / 2 + 1, multiplied (fmulmod_var, |.| < 0.6 q) in the
// evaluation order the forward leaves them in, and transformed back.  The
// register budget targets 2 CTAs of N / 16 threads per SM.
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, (NttShape<LOGN, K>::T >= 512 ? 1 : 512 / NttShape<LOGN, K>::T))
    k_poly_mul(u64* __restrict__ out, const u64* __restrict__ a, const u64* __restrict__ b,
               int n_polys, int n_limbs, int prime_begin, const PrimeInfo* __restrict__ pi,
               const TwD* __restrict__ tw, int cyclic) {
  extern __shared__ u64 sm[];
  using S = NttShape<LOGN, K>;
  const int limb = blockIdx.x / n_polys;  // limb-major, like k_ntt
  const long long poly = blockIdx.x % n_polys;
  const int pidx = prime_begin + limb;
  const PrimeInfo P = pi[pidx];
  const size_t off = ((size_t)poly * n_limbs + limb) * S::N;
  const TwD* tb = twbase<LOGN>(tw, pidx);
  const int tid = threadIdx.x;
  double x[S::E], y[S::E];
#pragma unroll
  for (int e = 0; e < S::E; ++e) x[e] = u2d(reduce_any(ld_stream(a + off + posC<LOGN, K>(tid, e)), P));
  ntt_fwd_d<LOGN, K>(x, sm, tid, tb, P, cyclic);
  __syncthreads();
#pragma unroll
  for (int e = 0; e < S::E; ++e) y[e] = u2d(reduce_any(ld_stream(b + off + posC<LOGN, K>(tid, e)), P));
  ntt_fwd_d<LOGN, K>(y, sm, tid, tb, P, cyclic);
#pragma unroll
  for (int e = 0; e < S::E; ++e)
    x[e] = fmulmod_var(dreduce(x[e], P.qd, P.qinv_d), dreduce(y[e], P.qd, P.qinv_d), P.qd, P.qinv_d);
  __syncthreads();
  u64 r[S::E];
  ntt_inv_d<LOGN, K>(x, r, sm, tid, tb, P, cyclic);
#pragma unroll
  for (int e = 0; e < S::E; ++e) out[off + posC<LOGN, K>(tid, e)] = r[e];
}

extern "C" int ckks_poly_mul(const ckks_ctx* ctx, uint64_t* out, const uint64_t* a,
                             const uint64_t* b, int n_polys, int prime_begin, int n_limbs,
                             int cyclic, void* stream) {
  if (int rc = check_limbs(ctx, prime_begin, n_limbs, "ckks_poly_mul")) return rc;
  if (!cyclic)
    for (int l = 0; l < n_limbs; ++l)
      CKKS_REQUIRE(ctx->has_nega[prime_begin + l],
                   "ckks_poly_mul: prime %d has no 2N-th root; use ckks_poly_mul_anyq",
                   prime_begin + l);
  if (n_polys <= 0) return CKKS_OK;
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    using S = NttShape<L, K>;
    auto kern = k_poly_mul<L, K>;
    ensure_smem(kern, S::SMEM_WORDS * 8);
    kern<<<grid1d((long long)n_polys * n_limbs), S::T, S::SMEM_WORDS * 8, as_stream(stream)>>>(
        reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(a),
        reinterpret_cast<const u64*>(b), n_polys, n_limbs, prime_begin, ctx->d_pi, ctx->d_tw, cyclic);
    return ckks_check_launch("ckks_poly_mul");
  });
}

// ------------------------------------------------------------------ any-q product
// Exact (a*b mod q) for arbitrary q < 2^50 with a, b < 2^50 (float quotient +
// wrapping remainder; the estimate is off by at most one in either direction).
__device__ __forceinline__ u64 mulmod_anyq(u64 a, u64 b, u64 q, double qd) {
  const double est = floor(__dmul_rn(__ull2double_rn(a), __ull2double_rn(b)) / qd);
  const u64 qt = (u64)est;
  i64 r = (i64)(a * b - qt * q);
  if (r < 0) r += (i64)q;
  if (r < 0) r += (i64)q;
  if (r >= (i64)q) r -= (i64)q;
  if (r >= (i64)q) r -= (i64)q;
  return (u64)r;
}

__device__ __forceinline__ u64 mod_anyq(u64 a, u64 q, double qd) { return mulmod_anyq(a, 1, q, qd); }

struct GarnerConsts {
  u64 p[3];
  TwPair p0inv_p1, p0inv_p2, p1inv_p2;
  u64 h[3];          // digits of (M - 1) / 2
  u64 q, p0_q, p0p1_q, m_q;
  double qd;
};

template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_poly_mul_anyq(u64* __restrict__ out, const u64* __restrict__ a, const u64* __restrict__ b,
                    const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw, int cyclic,
                    GarnerConsts G) {
  extern __shared__ u64 sm[];
  using S = NttShape<LOGN, K>;
  const long long poly = blockIdx.x;
  const size_t off = (size_t)poly * S::N;
  const int tid = threadIdx.x;
  u64 r[3][S::E];
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const PrimeInfo P = pi[k];
    const TwD* tb = twbase<LOGN>(tw, k);
    u64 x[S::E], y[S::E];
#pragma unroll
    for (int e = 0; e < S::E; ++e) x[e] = reduce_any(mod_anyq(a[off + posC<LOGN, K>(tid, e)], G.q, G.qd), P);
    ntt_fwd<LOGN, K>(x, sm, tid, tb, P, cyclic);
    __syncthreads();
#pragma unroll
    for (int e = 0; e < S::E; ++e) y[e] = reduce_any(mod_anyq(b[off + posC<LOGN, K>(tid, e)], G.q, G.qd), P);
    ntt_fwd<LOGN, K>(y, sm, tid, tb, P, cyclic);
#pragma unroll
    for (int e = 0; e < S::E; ++e) x[e] = mulmod(x[e], y[e], P);
    __syncthreads();
    ntt_inv<LOGN, K>(x, sm, tid, tb, P, cyclic);
    __syncthreads();
#pragma unroll
    for (int e = 0; e < S::E; ++e) r[k][e] = x[e];
  }
  const u64 p0 = G.p[0], p1 = G.p[1], p2 = G.p[2];
#pragma unroll
  for (int e = 0; e < S::E; ++e) {
    const u64 v0 = r[0][e];
    const u64 v0p1 = v0 % p1;
    const u64 v1 = shoup(submod(r[1][e], v0p1, p1), G.p0inv_p1.w, G.p0inv_p1.ws, p1);
    const u64 v0p2 = v0 % p2;
    const u64 t2 = shoup(submod(r[2][e], v0p2, p2), G.p0inv_p2.w, G.p0inv_p2.ws, p2);
    const u64 v2 = shoup(submod(t2, v1 % p2, p2), G.p1inv_p2.w, G.p1inv_p2.ws, p2);
    const bool neg = (v2 > G.h[2]) || (v2 == G.h[2] && (v1 > G.h[1] || (v1 == G.h[1] && v0 > G.h[0])));
    u64 s = mod_anyq(v0, G.q, G.qd);
    s = (s + mulmod_anyq(mod_anyq(v1, G.q, G.qd), G.p0_q, G.q, G.qd)) % G.q;
    s = (s + mulmod_anyq(mod_anyq(v2, G.q, G.qd), G.p0p1_q, G.q, G.qd)) % G.q;
    if (neg) s = (s + G.q - G.m_q) % G.q;
    out[off + posC<LOGN, K>(tid, e)] = s;
  }
  (void)p0;
}

extern "C" int ckks_poly_mul_anyq(const ckks_ctx* crt3, uint64_t* out, const uint64_t* a,
                                  const uint64_t* b, int n_polys, uint64_t q, int cyclic,
                                  void* stream) {
  CKKS_REQUIRE(crt3 != nullptr && crt3->n_primes == 3,
               "ckks_poly_mul_anyq: crt3 must be a context of exactly three primes");
  CKKS_REQUIRE(q >= 2 && q < (1ull << 45), "ckks_poly_mul_anyq: q outside [2, 2^45)");
  for (int k = 0; k < 3; ++k) {
    CKKS_REQUIRE(crt3->primes[k] > (1ull << 44), "ckks_poly_mul_anyq: CRT primes must exceed 2^44");
    if (!cyclic)
      CKKS_REQUIRE(crt3->has_nega[k], "ckks_poly_mul_anyq: CRT prime %d lacks a 2N-th root", k);
  }
  if (n_polys <= 0) return CKKS_OK;
  GarnerConsts G;
  const u64 p0 = crt3->primes[0], p1 = crt3->primes[1], p2 = crt3->primes[2];
  G.p[0] = p0;
  G.p[1] = p1;
  G.p[2] = p2;
  G.p0inv_p1 = h_twp(h_invmod(p0 % p1, p1), p1);
  G.p0inv_p2 = h_twp(h_invmod(p0 % p2, p2), p2);
  G.p1inv_p2 = h_twp(h_invmod(p1 % p2, p2), p2);
  G.h[0] = (p0 - 1) / 2;
  G.h[1] = (p1 - 1) / 2;
  G.h[2] = (p2 - 1) / 2;
  G.q = q;
  G.qd = (double)q;
  G.p0_q = p0 % q;
  G.p0p1_q = h_mulmod(p0 % q, p1 % q, q);
  G.m_q = h_mulmod(G.p0p1_q, p2 % q, q);
  return dispatch_logn(crt3->log_n, [&]<int L, int K>() -> int {
    using S = NttShape<L, K>;
    auto kern = k_poly_mul_anyq<L, K>;
    ensure_smem(kern, S::SMEM_WORDS * 8);
    kern<<<grid1d(n_polys), S::T, S::SMEM_WORDS * 8, as_stream(stream)>>>(
        reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(a),
        reinterpret_cast<const u64*>(b), crt3->d_pi, crt3->d_tw, cyclic, G);
    return ckks_check_launch("ckks_poly_mul_anyq");
  });
}

// ------------------------------------------------------------------ single-pair relin
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_relin_single(u64* __restrict__ f0, u64* __restrict__ f1, const u64* __restrict__ e0,
                   const u64* __restrict__ e1, const u64* __restrict__ e2,
                   const u64* __restrict__ ka, const u64* __restrict__ kb, int prime,
                   const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using S = NttShape<LOGN, K>;
  const size_t off = (size_t)blockIdx.x * S::N;
  const PrimeInfo P = pi[prime];
  const TwD* tb = twbase<LOGN>(tw, prime);
  const int tid = threadIdx.x;
  u64 x[S::E], y[S::E];
#pragma unroll
  for (int e = 0; e < S::E; ++e) x[e] = reduce_any(e2[off + posC<LOGN, K>(tid, e)], P);
  ntt_fwd<LOGN, K>(x, sm, tid, tb, P);
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    const u64* key = pass == 0 ? kb : ka;
    __syncthreads();
#pragma unroll
    for (int e = 0; e < S::E; ++e) y[e] = reduce_any(key[off + posC<LOGN, K>(tid, e)], P);
    ntt_fwd<LOGN, K>(y, sm, tid, tb, P);
#pragma unroll
    for (int e = 0; e < S::E; ++e) y[e] = mulmod(x[e], y[e], P);
    __syncthreads();
    ntt_inv<LOGN, K>(y, sm, tid, tb, P);
    const u64* ein = pass == 0 ? e0 : e1;
    u64* fo = pass == 0 ? f0 : f1;
#pragma unroll
    for (int e = 0; e < S::E; ++e) {
      const int p = posC<LOGN, K>(tid, e);
      const u64 base = ein[off + p];
      fo[off + p] = pass == 0 ? addmod(base, y[e], P.q) : submod(base, y[e], P.q);
    }
  }
}

extern "C" int ckks_relin_single(const ckks_ctx* ctx, uint64_t* f0, uint64_t* f1,
                                 const uint64_t* e0, const uint64_t* e1, const uint64_t* e2,
                                 const uint64_t* ka, const uint64_t* kb, int n_polys, int prime,
                                 void* stream) {
  if (int rc = check_limbs(ctx, prime, 1, "ckks_relin_single")) return rc;
  CKKS_REQUIRE(ctx->has_nega[prime], "ckks_relin_single: prime %d has no 2N-th root", prime);
  if (n_polys <= 0) return CKKS_OK;
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    using S = NttShape<L, K>;
    auto kern = k_relin_single<L, K>;
    ensure_smem(kern, S::SMEM_WORDS * 8);
    kern<<<grid1d(n_polys), S::T, S::SMEM_WORDS * 8, as_stream(stream)>>>(
        reinterpret_cast<u64*>(f0), reinterpret_cast<u64*>(f1), reinterpret_cast<const u64*>(e0),
        reinterpret_cast<const u64*>(e1), reinterpret_cast<const u64*>(e2),
        reinterpret_cast<const u64*>(ka), reinterpret_cast<const u64*>(kb), prime, ctx->d_pi,
        ctx->d_tw);
    return ckks_check_launch("ckks_relin_single");
  });
}

// ------------------------------------------------------------------ masked relin
// First-order masked single-pair relinearisation: the key (a, b) arrives as
// two additive shares (a1, b1), (a2, b2).  Each share is transformed,
// multiplied by NTT(e2) and brought back on its own; only the four
// coefficient-domain products are summed, so no register or buffer ever holds
// a1 + a2 or b1 + b2 (the two-pass schedule of rtl/m3/keyswitch_pipe_masked.sv:1-27):
//   f0 = e2 b1 + (e0 + e2 b2),   f1 = (e1 - e2 a1) - e2 a2.
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_relin_masked(u64* __restrict__ f0, u64* __restrict__ f1, const u64* __restrict__ e0,
                   const u64* __restrict__ e1, const u64* __restrict__ e2,
                   const u64* __restrict__ a1, const u64* __restrict__ b1,
                   const u64* __restrict__ a2, const u64* __restrict__ b2, int prime,
                   const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using S = NttShape<LOGN, K>;
  const size_t off = (size_t)blockIdx.x * S::N;
  const PrimeInfo P = pi[prime];
  const TwD* tb = twbase<LOGN>(tw, prime);
  const int tid = threadIdx.x;
  u64 x[S::E], y[S::E], acc[S::E];
#pragma unroll
  for (int e = 0; e < S::E; ++e) x[e] = reduce_any(e2[off + posC<LOGN, K>(tid, e)], P);
  ntt_fwd<LOGN, K>(x, sm, tid, tb, P);
#pragma unroll 1
  for (int out = 0; out < 2; ++out) {
#pragma unroll
    for (int e = 0; e < S::E; ++e)
      acc[e] = reduce_any((out == 0 ? e0 : e1)[off + posC<LOGN, K>(tid, e)], P);
#pragma unroll 1
    for (int share = 0; share < 2; ++share) {
      const u64* key = out == 0 ? (share == 0 ? b1 : b2) : (share == 0 ? a1 : a2);
      __syncthreads();
#pragma unroll
      for (int e = 0; e < S::E; ++e) y[e] = reduce_any(key[off + posC<LOGN, K>(tid, e)], P);
      ntt_fwd<LOGN, K>(y, sm, tid, tb, P);
#pragma unroll
      for (int e = 0; e < S::E; ++e) y[e] = mulmod(x[e], y[e], P);
      __syncthreads();
      ntt_inv<LOGN, K>(y, sm, tid, tb, P);
#pragma unroll
      for (int e = 0; e < S::E; ++e) acc[e] = out == 0 ? addmod(acc[e], y[e], P.q) : submod(acc[e], y[e], P.q);
    }
    u64* fo = out == 0 ? f0 : f1;
#pragma unroll
    for (int e = 0; e < S::E; ++e) fo[off + posC<LOGN, K>(tid, e)] = acc[e];
  }
}

extern "C" int ckks_relin_single_masked(const ckks_ctx* ctx, uint64_t* f0, uint64_t* f1,
                                        const uint64_t* e0, const uint64_t* e1, const uint64_t* e2,
                                        const uint64_t* a1, const uint64_t* b1, const uint64_t* a2,
                                        const uint64_t* b2, int n_polys, int prime, void* stream) {
  const char* fn = "ckks_relin_single_masked";
  if (int rc = check_limbs(ctx, prime, 1, fn)) return rc;
  CKKS_REQUIRE(ctx->has_nega[prime], "%s: prime %d has no 2N-th root", fn, prime);
  if (n_polys <= 0) return CKKS_OK;
  CKKS_REQUIRE(f0 && f1 && e0 && e1 && e2 && a1 && b1 && a2 && b2, "%s: NULL pointer argument", fn);
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    using S = NttShape<L, K>;
    auto kern = k_relin_masked<L, K>;
    ensure_smem(kern, S::SMEM_WORDS * 8);
    kern<<<grid1d(n_polys), S::T, S::SMEM_WORDS * 8, as_stream(stream)>>>(
        reinterpret_cast<u64*>(f0), reinterpret_cast<u64*>(f1), reinterpret_cast<const u64*>(e0),
        reinterpret_cast<const u64*>(e1), reinterpret_cast<const u64*>(e2),
        reinterpret_cast<const u64*>(a1), reinterpret_cast<const u64*>(b1),
        reinterpret_cast<const u64*>(a2), reinterpret_cast<const u64*>(b2), prime, ctx->d_pi,
        ctx->d_tw);
    return ckks_check_launch(fn);
  });
}
