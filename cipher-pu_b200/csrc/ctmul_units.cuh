// ctmul_units.cuh - the work units of the ct-mult's three kernels (and of
// the ct x pt + rescale kernel) as device functions: one call = one unit on
// one CTA of NttShape<LOGN, K>::T threads with the kernel's shared memory.
// The kernels in ctmul.cu / ctpt.cu loop over their units with these, and so
// does the persistent batch kernel (batch_persistent.cu), which runs units of
// every stage in one launch.  COH = true reads the intermediates written by
// other CTAs through the coherent L2 path (__ldcg): a unit may run in the same
// launch as the unit that produced them, so the read-only path must not hold
// a stale line; false (separate launches) keeps the read-only path.
#pragma once
#include "ntt.cuh"

struct CmScratch {
  u64* d01;   // [n_ct][2][level][N]  tensor d0, d1 (evaluation)
  u64* d2n;   // [n_ct][level][N]     tensor d2 (evaluation)
  u64* d2c;   // [n_ct][level][N]     d2 digits (coefficient)
  u64* acc;   // [n_ct][2][level][N]  key inner product over q_i (evaluation)
  u64* accp;  // [n_ct][2][N]         key inner product over p (evaluation)
};

// a load through L2 only (ld.global.cg: never a stale L1 line)
__device__ __forceinline__ u64 ld_l2(const u64* p) {
  u64 v;
  asm("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

// scratch loads, layout C
template <int LOGN, int K, bool COH>
__device__ __forceinline__ void load_sc(u64 (&x)[1 << K], const u64* __restrict__ src, int tid) {
  if constexpr (COH) {
#pragma unroll
    for (int e = 0; e < (1 << K); ++e) x[e] = ld_l2(src + posC<LOGN, K>(tid, e));
  } else {
    load_c<LOGN, K>(x, src, tid);
  }
}

// ---------------------------------------------------------------- tensor unit
// unit = j n_ct + ct: Karatsuba tensor of limb j of pair ct, its d2 INTT
// (the digit).  All global traffic is lane-contiguous (layout C); d2 is
// re-distributed to layout Z through shared memory for its INTT.
template <int LOGN, int K>
__device__ __forceinline__ void cm_tensor_unit(const u64* __restrict__ A, const u64* __restrict__ B,
                                               const CmScratch& S, int level, const PrimeInfo* __restrict__ pi,
                                               const TwD* __restrict__ tw, int n_ct, long long unit, u64* sm,
                                               int tid) {
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  const int j = unit / n_ct;  // limb-major: resident CTAs share q_j's tables
  const long long ct = unit % n_ct;
  const PrimeInfo P = pi[j];
  const size_t LN = (size_t)level * N;
  const u64* a0 = A + ct * 2 * LN + (size_t)j * N;
  const u64* b0 = B + ct * 2 * LN + (size_t)j * N;
  u64* d0 = S.d01 + ct * 2 * LN + (size_t)j * N;
  // Products in FP64 (exact two-product + rounded quotient, fmulmod_var):
  // d2 = a1 b1, d0 = a0 b0, d1 = (a0 + a1)(b0 + b1) - d0 - d2, each partial
  // result below 2^48 in magnitude, reduced to [0, q) once at the end.
  u64 x[Sh::E], y[Sh::E];
  load_c<LOGN, K>(x, a0 + LN, tid);
  load_c<LOGN, K>(y, b0 + LN, tid);
  double m2d[Sh::E];
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) m2d[e] = fmulmod_var(u2d(x[e]), u2d(y[e]), P.qd, P.qinv_d);
  u64 a0v[Sh::E], b0v[Sh::E];
  load_c<LOGN, K>(a0v, a0, tid);
  load_c<LOGN, K>(b0v, b0, tid);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) {
    const double a0d = u2d(a0v[e]), b0d = u2d(b0v[e]);
    const double m0 = fmulmod_var(a0d, b0d, P.qd, P.qinv_d);
    const double s1 = fmulmod_var(__dadd_rn(a0d, u2d(x[e])), __dadd_rn(b0d, u2d(y[e])), P.qd, P.qinv_d);
    a0v[e] = d2canon(m0, P.qd, P.qinv_d);
    b0v[e] = d2canon(__dadd_rn(__dadd_rn(s1, -m0), -m2d[e]), P.qd, P.qinv_d);  // |.| < 3 2^48
  }
  store_c<LOGN, K>(a0v, d0, tid);
  store_c<LOGN, K>(b0v, d0 + LN, tid);
  u64 m2[Sh::E];
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) m2[e] = d2canon(m2d[e], P.qd, P.qinv_d);
  store_c<LOGN, K>(m2, S.d2n + ct * LN + (size_t)j * N, tid);
  c_to_z<LOGN, K>(m2d, sm, tid);  // |m2d| < 0.6 q: straight into the FP64 inverse
  ntt_inv_d<LOGN, K>(m2d, m2, sm, tid, twbase<LOGN>(tw, j), P);
  store_c<LOGN, K>(m2, S.d2c + ct * LN + (size_t)j * N, tid);
}

// ---------------------------------------------------------------- ModUp unit
// unit = (level - i) n_ct + ct: target prime i (i = level: the special
// prime, first in the unit order) of pair ct.  Each digit is transformed
// (layout C in, Z out) and re-distributed to layout C, so the key limbs,
// stored in natural order, are read lane-contiguously.  The two accumulators
// live in thread-private shared-memory slots (index e * T + tid).
template <int LOGN, int K, bool COH>
__device__ __forceinline__ void cm_modup_unit(const CmScratch& S, const double* __restrict__ key, int level, int nq,
                                              const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw,
                                              int n_ct, long long unit, u64* sm, int tid) {
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  constexpr int T = Sh::T;
  u64* acc0s = sm + Sh::SMEM_WORDS;
  u64* acc1s = acc0s + N;
  // target-major (resident CTAs share one prime), special prime first: its
  // CTAs transform every digit, one more than the others, so they go first
  // and the shorter ones fill the last wave
  const int ti = level - (int)(unit / n_ct);
  const long long ct = unit % n_ct;
  const bool special = ti == level;
  const int pidx = special ? nq : ti;
  const PrimeInfo P = pi[pidx];
  const size_t LN = (size_t)level * N;
  const TwD* tb = twbase<LOGN>(tw, pidx);
  double* acc0s_d = reinterpret_cast<double*>(acc0s);
  double* acc1s_d = reinterpret_cast<double*>(acc1s);
#pragma unroll 1
  for (int j = 0; j < level; ++j) {
    // digit j as exact doubles in layout C: its evaluation-domain residues at
    // its own prime, else its coefficient residues (< q_j < 2 q_i) transformed
    // unreduced (|x| < 2^51 on return, fine for fmulmod)
    double x[Sh::E];
    u64 xu[Sh::E];
    if (!special && j == ti) {
      load_sc<LOGN, K, COH>(xu, S.d2n + ct * LN + (size_t)j * N, tid);
#pragma unroll
      for (int e = 0; e < Sh::E; ++e) x[e] = u2d(xu[e]);
    } else {
      load_sc<LOGN, K, COH>(xu, S.d2c + ct * LN + (size_t)j * N, tid);
#pragma unroll
      for (int e = 0; e < Sh::E; ++e) x[e] = u2d(xu[e]);
      ntt_fwd_d<LOGN, K>(x, sm, tid, tb, P);
      z_to_c<LOGN, K>(x, sm, tid);
    }
    // key inner product in exact FP64 on the key values alone (8 bytes per
    // word): w / q is formed as w * (1/q), two roundings off, so the quotient
    // estimate may miss by one and each product lands within 1.5 q (still
    // exact: every intermediate is an integer below 2^53); the running sum is
    // folded back below q / 2 + 1 every 16 digits so it stays exact
#pragma unroll 1
    for (int kk = 0; kk < 2; ++kk) {
      const double* kp = reinterpret_cast<const double*>(key) + (((size_t)j * 2 + kk) * (nq + 1) + pidx) * (2 * N);
      double* acc = kk ? acc1s_d : acc0s_d;
      const bool fold = (j & 15) == 15;
#pragma unroll
      for (int e = 0; e < Sh::E; ++e) {
        const double w = ld_stream_d(kp + posC<LOGN, K>(tid, e));
        const int s = e * T + tid;
        const double t = fmulmod(x[e], w, __dmul_rn(w, P.qinv_d), P.qd);
        double a = j == 0 ? t : __dadd_rn(acc[s], t);
        if (fold) {
          const double qt = __dadd_rn(__fma_rn(a, P.qinv_d, CKKS_FP_MAGIC), -CKKS_FP_MAGIC);
          a = __fma_rn(-qt, P.qd, a);
        }
        acc[s] = a;
      }
    }
  }
  // Special-prime accumulators stay in the evaluation domain here; kernel C
  // (one CTA per output polynomial) brings each back with one INTT, which
  // keeps the per-CTA work of this kernel within one transform of each other.
  u64 x[Sh::E];
  u64* o = special ? S.accp + ct * 2 * N : S.acc + ct * 2 * LN + (size_t)ti * N;
  const size_t kstride = special ? (size_t)N : LN;
#pragma unroll 1
  for (int k = 0; k < 2; ++k) {
    const u64* a = k ? acc1s : acc0s;
#pragma unroll
    for (int e = 0; e < Sh::E; ++e)
      x[e] = d2canon(reinterpret_cast<const double*>(a)[e * T + tid], P.qd, P.qinv_d);
    store_c<LOGN, K>(x, o + (size_t)k * kstride, tid);
  }
}

// ---------------------------------------------------------------- ModDown + rescale unit
// unit = 2 ct + k: output polynomial k of pair ct.
template <int LOGN, int K, bool COH>
__device__ __forceinline__ void cm_down_unit(const CmScratch& S, u64* __restrict__ out, int level, int nq,
                                             const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw,
                                             const TwPair* __restrict__ pinv, const TwPair* __restrict__ qtinv,
                                             long long unit, u64* sm, int tid) {
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  constexpr int T = Sh::T;
  double* vs = reinterpret_cast<double*>(sm + Sh::SMEM_WORDS);
  double* ws = vs + N;
  const long long ct = unit >> 1;
  const int k = unit & 1;
  const int t = level - 1;
  const size_t LN = (size_t)level * N;
  const PrimeInfo PP = pi[nq];
  const PrimeInfo PT = pi[t];
  const u64* dk = S.d01 + ct * 2 * LN + (size_t)k * LN;
  const u64* ak = S.acc + ct * 2 * LN + (size_t)k * LN;
  u64* ok = out + ((size_t)ct * 2 + k) * (size_t)t * N;

  double d[Sh::E];
  u64 x[Sh::E];
  // d_k's limbs (read after this unit's first transform) toward L2 now: the
  // tensor kernel wrote them long before and, with four sub-batches in
  // flight, they may have left L2 (measured +0.4 % on the whole step at
  // N = 2^12, L = 3; prefetching the accumulators as well lost 0.3 %).  The
  // per-shape kernel only: in the persistent batch kernel (COH) the loop
  // costs registers that its N = 2^13 units spill.
  if constexpr (!COH) {
#pragma unroll 1
    for (int i = 0; i <= t; ++i) {
#pragma unroll
      for (int e = 0; e < Sh::E; ++e)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(dk + (size_t)i * N + posC<LOGN, K>(tid, e)));
    }
  }
  load_sc<LOGN, K, COH>(x, S.accp + (ct * 2 + k) * N, tid);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) d[e] = u2d(x[e]);
  c_to_z<LOGN, K>(d, sm, tid);
  ntt_inv_d<LOGN, K>(d, x, sm, tid, twbase<LOGN>(tw, nq), PP);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) vs[e * T + tid] = x[e] > PP.half ? u2d(x[e]) - PP.qd : u2d(x[e]);
  // Rescale limb t in the coefficient domain without a transform of v:
  // w = INTT_t(d_t + acc_t p^-1) - v p^-1, equal mod q_t to
  // INTT_t(d_t + (acc_t - NTT_t([v]_t)) p^-1) by linearity of the NTT.
  const double ptw = (double)pinv[t].w;
  const double ptq = __ddiv_rn(ptw, PT.qd);
  {
    u64 dv[Sh::E];
    load_sc<LOGN, K, COH>(dv, dk + (size_t)t * N, tid);
    load_sc<LOGN, K, COH>(x, ak + (size_t)t * N, tid);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const double dc = dv[e] > PT.half ? u2d(dv[e]) - PT.qd : u2d(dv[e]);
      d[e] = __dadd_rn(fmulmod(u2d(x[e]), ptw, ptq, PT.qd), dc);
    }
  }
  c_to_z<LOGN, K>(d, sm, tid);
  ntt_inv_d<LOGN, K>(d, x, sm, tid, twbase<LOGN>(tw, t), PT);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) {
    const u64 w = d2canon(__dadd_rn(u2d(x[e]), -fmulmod(vs[e * T + tid], ptw, ptq, PT.qd)), PT.qd, PT.qinv_d);
    ws[e * T + tid] = w > PT.half ? u2d(w) - PT.qd : u2d(w);
  }
#pragma unroll 1
  for (int i = 0; i < t; ++i) {
    const PrimeInfo P = pi[i];
    const double pvw = (double)pinv[i].w;
    const double pvq = __ddiv_rn(pvw, P.qd);
    const double ciw = (double)qtinv[(size_t)t * nq + i].w;
    const double ciq = __ddiv_rn(ciw, P.qd);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e)
      d[e] = __dadd_rn(fmulmod(vs[e * T + tid], pvw, pvq, P.qd), ws[e * T + tid]);  // |.| < 2 q_i
    ntt_fwd_d<LOGN, K>(d, sm, tid, twbase<LOGN>(tw, i), P);
    z_to_c<LOGN, K>(d, sm, tid);
    u64 dv[Sh::E], av[Sh::E];
    load_sc<LOGN, K, COH>(dv, dk + (size_t)i * N, tid);
    load_sc<LOGN, K, COH>(av, ak + (size_t)i * N, tid);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const double sd = __dadd_rn(__dadd_rn(u2d(dv[e]), fmulmod(u2d(av[e]), pvw, pvq, P.qd)), -d[e]);
      x[e] = d2canon(fmulmod(sd, ciw, ciq, P.qd), P.qd, P.qinv_d);
    }
    store_c<LOGN, K>(x, ok + (size_t)i * N, tid);
  }
}

// ---------------------------------------------------------------- ct x pt + rescale unit
// Output polynomial k of ciphertext c: x_i = a_k,i * p_i per limb (evaluation
// domain); the last limb is brought to the coefficient domain (INTT),
// centred, and for every remaining limb out_i = (x_i - NTT_i([w]_{q_i})) *
// q_t^-1.  Reads only the caller's inputs, so it has no coherent variant.
template <int LOGN, int K>
__device__ __forceinline__ void ctpt_unit(u64* __restrict__ out, const u64* __restrict__ ct,
                                          const u64* __restrict__ pt, int pt_stride, int level,
                                          const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw,
                                          const TwPair* __restrict__ qtinv, int nq, long long c, int k, u64* sm,
                                          int tid) {
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  constexpr int T = Sh::T;
  double* ws = reinterpret_cast<double*>(sm + Sh::SMEM_WORDS);
  const int t = level - 1;
  const size_t LN = (size_t)level * N;
  const u64* a = ct + (c * 2 + k) * LN;
  const u64* p = pt + (size_t)c * pt_stride * LN;
  u64* o = out + (c * 2 + k) * (size_t)t * N;
  const PrimeInfo PT = pi[t];
  // FP64 throughout: products by fmulmod_var (|.| < 0.6 q), the rescale limb
  // w kept centred and signed (|w| <= q_t / 2 < q_i), q_t^-1 by fmulmod.
  double d[Sh::E];
  u64 x[Sh::E], y[Sh::E];
  load_c<LOGN, K>(x, a + (size_t)t * N, tid);
  load_c<LOGN, K>(y, p + (size_t)t * N, tid);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) d[e] = fmulmod_var(u2d(x[e]), u2d(y[e]), PT.qd, PT.qinv_d);
  c_to_z<LOGN, K>(d, sm, tid);
  ntt_inv_d<LOGN, K>(d, x, sm, tid, twbase<LOGN>(tw, t), PT);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) ws[e * T + tid] = x[e] > PT.half ? u2d(x[e]) - PT.qd : u2d(x[e]);
#pragma unroll 1
  for (int i = 0; i < t; ++i) {
    const PrimeInfo P = pi[i];
    const double ciw = (double)qtinv[(size_t)t * nq + i].w;
    const double ciq = __ddiv_rn(ciw, P.qd);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) d[e] = ws[e * T + tid];
    ntt_fwd_d<LOGN, K>(d, sm, tid, twbase<LOGN>(tw, i), P);  // |d| < 13.75 q
    z_to_c<LOGN, K>(d, sm, tid);
    load_c<LOGN, K>(x, a + (size_t)i * N, tid);
    load_c<LOGN, K>(y, p + (size_t)i * N, tid);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) {
      const double sd = __dadd_rn(fmulmod_var(u2d(x[e]), u2d(y[e]), P.qd, P.qinv_d), -d[e]);
      x[e] = d2canon(fmulmod(sd, ciw, ciq, P.qd), P.qd, P.qinv_d);
    }
    store_c<LOGN, K>(x, o + (size_t)i * N, tid);
  }
}
