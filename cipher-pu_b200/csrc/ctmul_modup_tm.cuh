// ctmul_modup_tm.cuh - the ct-mult's ModUp + key inner product with its two
// accumulators in Tensor Memory instead of shared memory.
//
// The shared-memory ModUp (cm_modup_unit) keeps, per thread, 2 x E running
// sums as doubles in shared memory next to the transform buffer: at
// N = 2^12 that is 64 KB of accumulators + 34 KB of transform buffer per
// CTA, so only two 256-thread CTAs fit an SM (16 warps).  Here the sums live
// in TMEM (4 E 32-bit cells per thread: 128 columns for a 256-thread CTA),
// the CTA needs only the transform buffer, and with an 85-register budget
// three CTAs share an SM (24 warps, 3 x 128 of the 512 TMEM columns).
// Arithmetic and results are those of cm_modup_unit, value for value.
#pragma once
#include "ctmul_units.cuh"
#include "tmem.cuh"

template <int LOGN, int K>
struct ModupTm {
  using Sh = NttShape<LOGN, K>;
  static constexpr int E = Sh::E;
  static constexpr int CELLS = 4 * E;  // 2 accumulators x E doubles x 2 cells
  static constexpr uint32_t COLS = tmem_cols_for(Sh::T, CELLS);
  // resident threads per SM targeted (24 warps), as CTAs per SM
  static constexpr int MINB = 768 / Sh::T;
  // built where it was measured faster (N = 2^12: 1.43M against 1.39M
  // ct-mult/s at L = 3, 685K against 648K at L = 5; at N = 2^11 it lost 6 %)
  // and the target occupancy fits the SM's 512 TMEM columns
  static constexpr bool BUILT = K == 4 && LOGN == 12 && MINB * COLS <= 512;
};

// This thread's TMEM address of cell column 0: its warp's lane quarter
// (lanes 32 (w mod 4) ..), its 128-thread group's column range.
__device__ __forceinline__ uint32_t modup_tm_addr(uint32_t base, int tid, int cells) {
  return base + ((uint32_t)(((tid >> 5) & 3) * 32) << 16) + (uint32_t)((tid >> 7) * cells);
}

// One ModUp unit (unit = (level - i) n_ct + ct: target prime i of pair ct,
// i = level the special prime), accumulators at TMEM address ta: sum k,
// values 8 c .. 8 c + 7 at columns k 2E + 16 c.
template <int LOGN, int K>
__device__ __forceinline__ void cm_modup_unit_tm(const CmScratch& S, const double* __restrict__ key, int level,
                                                 int nq, const PrimeInfo* __restrict__ pi,
                                                 const TwD* __restrict__ tw, int n_ct, long long unit, u64* sm,
                                                 int tid, uint32_t ta) {
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  constexpr int E = Sh::E;
  const int ti = level - (int)(unit / n_ct);
  const long long ct = unit % n_ct;
  const bool special = ti == level;
  const int pidx = special ? nq : ti;
  const PrimeInfo P = pi[pidx];
  const size_t LN = (size_t)level * N;
  const TwD* tb = twbase<LOGN>(tw, pidx);
#pragma unroll 1
  for (int j = 0; j < level; ++j) {
    {
      // bring the first key polynomial's limb for this digit toward L1 while
      // the digit is transformed (both polynomials' limbs here, 3 CTAs x 64 KB,
      // would not fit the L1 left beside the shared memory: measured +1-1.6 %
      // for the first alone, +0.7-1 % for both; the second follows below)
      const double* kp = key + ((size_t)j * 2 * (nq + 1) + pidx) * (2 * N);
#pragma unroll
      for (int e = 0; e < E; ++e) asm volatile("prefetch.global.L1 [%0];" ::"l"(kp + posC<LOGN, K>(tid, e)));
    }
    double x[E];
    u64 xu[E];
    if (!special && j == ti) {
      load_c<LOGN, K>(xu, S.d2n + ct * LN + (size_t)j * N, tid);
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = u2d(xu[e]);
    } else {
      load_c<LOGN, K>(xu, S.d2c + ct * LN + (size_t)j * N, tid);
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = u2d(xu[e]);
      ntt_fwd_d<LOGN, K>(x, sm, tid, tb, P);
      z_to_c<LOGN, K>(x, sm, tid);
    }
    const bool fold = (j & 15) == 15;
#pragma unroll 1
    for (int kk = 0; kk < 2; ++kk) {
      const double* kp = key + (((size_t)j * 2 + kk) * (nq + 1) + pidx) * (2 * N);
      if (kk == 0) {
        // and the second polynomial's limb while the first one's products run
        // (by then the first limb's lines are in use; both at the digit's
        // start would not fit the L1 beside the shared memory)
        const double* kp1 = kp + (size_t)(nq + 1) * (2 * N);
#pragma unroll
        for (int e = 0; e < E; ++e) asm volatile("prefetch.global.L1 [%0];" ::"l"(kp1 + posC<LOGN, K>(tid, e)));
      }
#pragma unroll
      for (int c = 0; c < E / 8; ++c) {
        const uint32_t addr = ta + (uint32_t)(kk * 2 * E + 16 * c);
        double a8[8];
        if (j) tmem_ld8(addr, a8);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int e = 8 * c + i;
          const double w = ld_stream_d(kp + posC<LOGN, K>(tid, e));
          const double t = fmulmod(x[e], w, __dmul_rn(w, P.qinv_d), P.qd);
          double a = j == 0 ? t : __dadd_rn(a8[i], t);
          if (fold) {
            const double qt = __dadd_rn(__fma_rn(a, P.qinv_d, CKKS_FP_MAGIC), -CKKS_FP_MAGIC);
            a = __fma_rn(-qt, P.qd, a);
          }
          a8[i] = a;
        }
        tmem_st8(addr, a8);
      }
    }
  }
  u64 xo[E];
  u64* o = special ? S.accp + ct * 2 * N : S.acc + ct * 2 * LN + (size_t)ti * N;
  const size_t kstride = special ? (size_t)N : LN;
#pragma unroll 1
  for (int k = 0; k < 2; ++k) {
#pragma unroll
    for (int c = 0; c < E / 8; ++c) {
      double a8[8];
      tmem_ld8(ta + (uint32_t)(k * 2 * E + 16 * c), a8);
#pragma unroll
      for (int i = 0; i < 8; ++i) xo[8 * c + i] = d2canon(a8[i], P.qd, P.qinv_d);
    }
    store_c<LOGN, K>(xo, o + (size_t)k * kstride, tid);
  }
}

// The kernel: `upc` consecutive units per CTA; one warp allocates the
// CTA's columns before the first and frees them after the last.
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, ModupTm<LOGN, K>::MINB)
    k_cm_modup_tm(CmScratch S, const double* __restrict__ key, int level, int nq, const PrimeInfo* __restrict__ pi,
                  const TwD* __restrict__ tw, int n_ct, long long n_units, int upc) {
  using M = ModupTm<LOGN, K>;
  extern __shared__ u64 sm[];
  __shared__ uint32_t s_tbase;
  const int tid = threadIdx.x;
  if (tid < 32) tmem_alloc_warp(&s_tbase, M::COLS);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t ta = modup_tm_addr(s_tbase, tid, M::CELLS);
  for (int r = 0; r < upc; ++r) {
    const long long unit = (long long)blockIdx.x * upc + r;
    if (unit >= n_units) break;  // uniform across the CTA
    if (r) __syncthreads();      // the previous unit is done with shared memory
    cm_modup_unit_tm<LOGN, K>(S, key, level, nq, pi, tw, n_ct, unit, sm, tid, ta);
  }
  tmem_fence_before_sync();
  __syncthreads();
  if (tid < 32) tmem_dealloc_warp(s_tbase, M::COLS);
}
