// ctmul.cu - batched CKKS homomorphic multiply with hybrid relinearisation
// and RNS rescale (the ct-mult + relin + rescale hot path).
//
// Data flow for n_ct ciphertext pairs at `level` limbs q_0..q_{t} (t = level-1)
// and one special prime p, dnum = level digits (one limb per digit):
//
//   A  tensor    (ct, j):  d0 = a0 b0, d2 = a1 b1, d1 = (a0+a1)(b0+b1) - d0 - d2
//                          (Karatsuba), d2 -> INTT_j -> coefficient digit j.
//   B  modup+ip  (ct, i):  for target prime i in {q_0..q_t, p}:
//                          acc_k = sum_j NTT_i([digit_j]_{q_i}) * ksk[j][k][i]
//                          (digit j at its own prime reuses the NTT-domain d2);
//                          the special-prime CTA also INTTs acc_0, acc_1.
//   C  moddown+rescale (ct, k):
//                          v = centred(acc_k mod p)            (coefficient)
//                          limb t : o_t = d_k,t + (acc_k,t - NTT_t([v]_t)) p^-1
//                                   w = centred(INTT_t(o_t))
//                          limb i<t: out = (d_k,i + acc_k,i p^-1
//                                           - NTT_i([v]_i p^-1 + [w]_i)) q_t^-1
//                          (ModDown and rescale conversions merged into one
//                          NTT per limb by linearity; bit-identical to doing
//                          them one after the other).
// Transforms per ct-mult at level L: L + (L-1)L + (L + 2) + 2(L + 1)
// = 22 at L = 3 (vs 26 for the unmerged sequence).
#include "dispatch.cuh"
#include "profile.hpp"

struct CmScratch {
  u64* d01;   // [n_ct][2][level][N]  tensor d0, d1 (evaluation)
  u64* d2n;   // [n_ct][level][N]     tensor d2 (evaluation)
  u64* d2c;   // [n_ct][level][N]     d2 digits (coefficient)
  u64* acc;   // [n_ct][2][level][N]  key inner product over q_i (evaluation)
  u64* accp;  // [n_ct][2][N]         key inner product over p (coefficient)
};

static size_t cm_words(int n, int n_ct, int level) {
  return (size_t)n_ct * n * (size_t)(6 * level + 2);
}

static CmScratch cm_carve(void* base, int n, int n_ct, int level) {
  CmScratch s;
  u64* p = reinterpret_cast<u64*>(base);
  const size_t ln = (size_t)level * n;
  s.d01 = p;
  p += (size_t)n_ct * 2 * ln;
  s.d2n = p;
  p += (size_t)n_ct * ln;
  s.d2c = p;
  p += (size_t)n_ct * ln;
  s.acc = p;
  p += (size_t)n_ct * 2 * ln;
  s.accp = p;
  return s;
}

// ---------------------------------------------------------------- kernel A
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_cm_tensor(const u64* __restrict__ A, const u64* __restrict__ B, CmScratch S, int level,
                const PrimeInfo* __restrict__ pi, const TwPair* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  const long long ct = blockIdx.x / level;
  const int j = blockIdx.x % level;
  const int tid = threadIdx.x;
  const PrimeInfo P = pi[j];
  const size_t LN = (size_t)level * N;
  const u64* a0 = A + ct * 2 * LN + (size_t)j * N;
  const u64* a1 = a0 + LN;
  const u64* b0 = B + ct * 2 * LN + (size_t)j * N;
  const u64* b1 = b0 + LN;
  u64* d0 = S.d01 + ct * 2 * LN + (size_t)j * N;
  u64* d1 = d0 + LN;
  u64* d2n = S.d2n + ct * LN + (size_t)j * N;
  u64* d2c = S.d2c + ct * LN + (size_t)j * N;
  u64 x[Sh::E];
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) {
    const int p = posZ<LOGN, K>(tid, e);
    const u64 A0 = a0[p], A1 = a1[p], B0 = b0[p], B1 = b1[p];
    const u64 m0 = mulmod(A0, B0, P);
    const u64 m2 = mulmod(A1, B1, P);
    u64 m1 = mulmod(addmod(A0, A1, P.q), addmod(B0, B1, P.q), P);
    m1 = submod(submod(m1, m0, P.q), m2, P.q);
    d0[p] = m0;
    d1[p] = m1;
    d2n[p] = m2;
    x[e] = m2;
  }
  ntt_inv<LOGN, K>(x, sm, tid, tw + ((size_t)j * 4 + TW_INV) * N, P);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) d2c[posC<LOGN, K>(tid, e)] = x[e];
}

// ---------------------------------------------------------------- kernel B
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_cm_modup(CmScratch S, const ulonglong2* __restrict__ key, int level, int nq,
               const PrimeInfo* __restrict__ pi, const TwPair* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  const long long ct = blockIdx.x / (level + 1);
  const int ti = blockIdx.x % (level + 1);
  const bool special = ti == level;
  const int pidx = special ? nq : ti;
  const int tid = threadIdx.x;
  const PrimeInfo P = pi[pidx];
  const size_t LN = (size_t)level * N;
  const TwPair* tf = tw + ((size_t)pidx * 4 + TW_FWD) * N;
  u64 acc0[Sh::E], acc1[Sh::E];
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) acc0[e] = acc1[e] = 0;
#pragma unroll 1
  for (int j = 0; j < level; ++j) {
    u64 x[Sh::E];
    if (!special && j == ti) {
      const u64* src = S.d2n + ct * LN + (size_t)j * N;
#pragma unroll
      for (int e = 0; e < Sh::E; ++e) x[e] = src[posZ<LOGN, K>(tid, e)];
    } else {
      const u64* src = S.d2c + ct * LN + (size_t)j * N;
#pragma unroll
      for (int e = 0; e < Sh::E; ++e) x[e] = csub(src[posC<LOGN, K>(tid, e)], P.q);
      ntt_fwd_lazy<LOGN, K>(x, sm, tid, tf, P.q, P.q2);
    }
    const ulonglong2* k0 = key + (((size_t)j * 2 + 0) * (nq + 1) + pidx) * N;
    const ulonglong2* k1 = key + (((size_t)j * 2 + 1) * (nq + 1) + pidx) * N;
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const int p = posZ<LOGN, K>(tid, e);
      const ulonglong2 w0 = __ldg(k0 + p);
      const ulonglong2 w1 = __ldg(k1 + p);
      acc0[e] += shoup_lazy(x[e], w0.x, w0.y, P.q);
      acc1[e] += shoup_lazy(x[e], w1.x, w1.y, P.q);
    }
  }
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) {
    acc0[e] = reduce_any(acc0[e], P);
    acc1[e] = reduce_any(acc1[e], P);
  }
  if (special) {
    const TwPair* ti_tab = tw + ((size_t)pidx * 4 + TW_INV) * N;
    u64* o0 = S.accp + ct * 2 * N;
    u64* o1 = o0 + N;
    ntt_inv<LOGN, K>(acc0, sm, tid, ti_tab, P);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) o0[posC<LOGN, K>(tid, e)] = acc0[e];
    ntt_inv<LOGN, K>(acc1, sm, tid, ti_tab, P);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) o1[posC<LOGN, K>(tid, e)] = acc1[e];
  } else {
    u64* o0 = S.acc + ct * 2 * LN + (size_t)ti * N;
    u64* o1 = o0 + LN;
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const int p = posZ<LOGN, K>(tid, e);
      o0[p] = acc0[e];
      o1[p] = acc1[e];
    }
  }
}

// ---------------------------------------------------------------- kernel C
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_cm_down(CmScratch S, u64* __restrict__ out, int level, int nq,
              const PrimeInfo* __restrict__ pi, const TwPair* __restrict__ tw,
              const TwPair* __restrict__ pinv, const TwPair* __restrict__ qtinv) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  const long long ct = blockIdx.x >> 1;
  const int k = blockIdx.x & 1;
  const int t = level - 1;
  const int tid = threadIdx.x;
  const size_t LN = (size_t)level * N;
  const PrimeInfo PP = pi[nq];
  const PrimeInfo PT = pi[t];
  const u64* accp = S.accp + (ct * 2 + k) * N;
  const u64* dk = S.d01 + ct * 2 * LN + (size_t)k * LN;
  const u64* ak = S.acc + ct * 2 * LN + (size_t)k * LN;
  u64* ok = out + ((size_t)ct * 2 + k) * (size_t)t * N;

  u64 v[Sh::E], x[Sh::E];
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) {
    v[e] = accp[posC<LOGN, K>(tid, e)];
    x[e] = v[e] > PP.half ? v[e] - PP.q + PT.q : v[e];
  }
  ntt_fwd_lazy<LOGN, K>(x, sm, tid, tw + ((size_t)t * 4 + TW_FWD) * N, PT.q, PT.q2);
  {
    const TwPair pt = pinv[t];
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const int p = posZ<LOGN, K>(tid, e);
      const u64 ks = shoup(ak[(size_t)t * N + p] + PT.q4 - x[e], pt.w, pt.ws, PT.q);
      x[e] = addmod(dk[(size_t)t * N + p], ks, PT.q);
    }
  }
  ntt_inv<LOGN, K>(x, sm, tid, tw + ((size_t)t * 4 + TW_INV) * N, PT);
#pragma unroll 1
  for (int i = 0; i < t; ++i) {
    const PrimeInfo P = pi[i];
    const TwPair pv = pinv[i];
    const TwPair ci = qtinv[(size_t)t * nq + i];
    u64 z[Sh::E];
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const u64 vi = v[e] > PP.half ? v[e] - PP.q + P.q : v[e];
      const u64 wi = x[e] > PT.half ? x[e] - PT.q + P.q : x[e];
      z[e] = shoup_lazy(vi, pv.w, pv.ws, P.q) + wi;  // [0, 3q)
    }
    ntt_fwd_lazy<LOGN, K>(z, sm, tid, tw + ((size_t)i * 4 + TW_FWD) * N, P.q, P.q2);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const int p = posZ<LOGN, K>(tid, e);
      const u64 s = dk[(size_t)i * N + p] + shoup_lazy(ak[(size_t)i * N + p], pv.w, pv.ws, P.q) +
                    P.q4 - z[e];  // (0, 7q)
      ok[(size_t)i * N + p] = shoup(s, ci.w, ci.ws, P.q);
    }
  }
}

// ---------------------------------------------------------------- key prep
__global__ void k_key_prepare(ulonglong2* __restrict__ out, const u64* __restrict__ in,
                              long long total, int log_n, int nlimb,
                              const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int limb = (int)((idx >> log_n) % nlimb);
  const PrimeInfo P = pi[limb];
  const u64 w = in[idx] % P.q;
  // floor(w 2^64 / q) = w * floor(2^64 / q) + floor(w (2^64 mod q) / q)
  const u64 num_lo = w * P.r_mod;
  u64 qt = (u64)floor(__dmul_rn(__ull2double_rn(w), __ull2double_rn(P.r_mod)) * P.qinv_d);
  i64 rem = (i64)(num_lo - qt * P.q);
  for (int it = 0; it < 3 && rem < 0; ++it) { rem += (i64)P.q; --qt; }
  for (int it = 0; it < 3 && rem >= (i64)P.q; ++it) { rem -= (i64)P.q; ++qt; }
  out[idx] = make_ulonglong2(w, w * P.one_s + qt);
}

extern "C" int ckks_relin_key_prepare(const ckks_ctx* ctx, uint64_t* prepared,
                                      const uint64_t* ksk, void* stream) {
  CKKS_REQUIRE(ctx != nullptr, "ckks_relin_key_prepare: ctx is NULL");
  CKKS_REQUIRE(ctx->n_special == 1, "ckks_relin_key_prepare: context needs one special prime");
  const long long total = (long long)ctx->n_q * 2 * ctx->n_primes * ctx->n;
  k_key_prepare<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<ulonglong2*>(prepared), reinterpret_cast<const u64*>(ksk), total,
      ctx->log_n, ctx->n_primes, ctx->d_pi);
  return ckks_check_launch("ckks_relin_key_prepare");
}

extern "C" size_t ckks_ct_mul_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level) {
  if (!ctx || n_ct < 0 || level < 1) return 0;
  return cm_words(ctx->n, n_ct, level) * sizeof(u64);
}

int ckks_ct_mul_launch(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                       const uint64_t* ct_b, const uint64_t* key, int n_ct, int level,
                       void* scratch, size_t scratch_bytes, void* stream, const char* fn) {
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(ctx->n_special == 1, "%s: context needs exactly one special prime", fn);
  CKKS_REQUIRE(level >= 2 && level <= ctx->n_q, "%s: level=%d outside [2, %d]", fn, level,
               ctx->n_q);
  CKKS_REQUIRE(ctx->log_n >= 5, "%s: log_n=%d below the supported minimum 5", fn, ctx->log_n);
  CKKS_REQUIRE(n_ct >= 0, "%s: n_ct < 0", fn);
  u64 pmin = ~0ull, pmax = 0;
  for (int i = 0; i < ctx->n_primes; ++i) {
    CKKS_REQUIRE(ctx->has_nega[i], "%s: prime %d has no 2N-th root", fn, i);
    pmin = ctx->primes[i] < pmin ? ctx->primes[i] : pmin;
    pmax = ctx->primes[i] > pmax ? ctx->primes[i] : pmax;
  }
  CKKS_REQUIRE(pmax < 2 * pmin && pmax < (1ull << 61) / 4,
               "%s: primes must satisfy max < 2 min (centred basis conversion)", fn);
  if (n_ct == 0) return CKKS_OK;
  CKKS_REQUIRE(out && ct_a && ct_b && key && scratch, "%s: NULL pointer argument", fn);
  const size_t need = ckks_ct_mul_scratch_bytes(ctx, n_ct, level);
  CKKS_REQUIRE(scratch_bytes >= need, "%s: scratch of %zu bytes < %zu needed", fn, scratch_bytes,
               need);
  CmScratch S = cm_carve(scratch, ctx->n, n_ct, level);
  cudaStream_t st = as_stream(stream);
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    if constexpr (L < 5) {
      return ckks_set_error(CKKS_EUNSUPPORTED, "%s: log_n too small", fn);
    } else {
      using Sh = NttShape<L, K>;
      const int smem = Sh::SMEM_WORDS * 8;
      auto ka = k_cm_tensor<L, K>;
      auto kb = k_cm_modup<L, K>;
      auto kc = k_cm_down<L, K>;
      ensure_smem(ka, smem);
      ensure_smem(kb, smem);
      ensure_smem(kc, smem);
      {
        ProfSpan span(CKKS_STAGE_CM_TENSOR, st);
        ka<<<grid1d((long long)n_ct * level), Sh::T, smem, st>>>(
            reinterpret_cast<const u64*>(ct_a), reinterpret_cast<const u64*>(ct_b), S, level,
            ctx->d_pi, ctx->d_tw);
      }
      if (int rc = ckks_check_launch(fn)) return rc;
      {
        ProfSpan span(CKKS_STAGE_CM_MODUP, st);
        kb<<<grid1d((long long)n_ct * (level + 1)), Sh::T, smem, st>>>(
            S, reinterpret_cast<const ulonglong2*>(key), level, ctx->n_q, ctx->d_pi, ctx->d_tw);
      }
      if (int rc = ckks_check_launch(fn)) return rc;
      {
        ProfSpan span(CKKS_STAGE_CM_DOWN, st);
        kc<<<grid1d((long long)n_ct * 2), Sh::T, smem, st>>>(
            S, reinterpret_cast<u64*>(out), level, ctx->n_q, ctx->d_pi, ctx->d_tw, ctx->d_pinv,
            ctx->d_qtinv);
      }
      return ckks_check_launch(fn);
    }
  });
}

extern "C" int ckks_ct_mul_relin_rescale(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                                         const uint64_t* ct_b, const uint64_t* key, int n_ct,
                                         int level, void* scratch, size_t scratch_bytes,
                                         void* stream) {
  return ckks_ct_mul_launch(ctx, out, ct_a, ct_b, key, n_ct, level, scratch, scratch_bytes, stream,
                            "ckks_ct_mul_relin_rescale");
}
