// ctmul_fused.cu - the ct-mult + relin + rescale of one ciphertext pair in one
// thread-block cluster, with no global scratch.
//
// A pair at `level` limbs q_0..q_t (t = level - 1) with one special prime p is
// handled by a cluster of level + 1 CTAs: CTA r < level owns prime q_r, CTA
// level owns p.  What the three-kernel path hands over through 640 KB of
// global scratch per pair (tensor digits, key inner products, ModDown
// conversions) moves here between the CTAs' shared memories (distributed
// shared memory, DSMEM), published in one buffer per CTA and read by the
// others after a cluster barrier.
//
//   stage A  CTA r < level: d0, d1, d2 = tensor product of limb r (Karatsuba,
//            FP64); the accumulators start as acc_k = d_k [p]_{q_r} +
//            d2 * ksk[r][k][r] (the digit at its own prime needs no
//            transform; folding d_k in as d_k p makes the later ModDown
//            (acc_k p^-1) produce d_k + ks_k directly); digit r = INTT_r(d2)
//            is published.  CTA p starts from zero.
//   B1 ----  digits visible cluster-wide
//   stage B  every CTA: for each digit j != r read from CTA j's buffer,
//            NTT to its own prime, acc_k += NTT(digit_j) * ksk[j][k][r].
//   B2 ----  digits consumed (buffers free)
//   stage C  per output polynomial k = 0, 1 (k = 1 overlapping the outputs of
//            k = 0):  CTA p publishes v_k = centred INTT_p(acc_k,p); CTA t
//            publishes u_k = INTT_t(acc_k,t p^-1); every CTA i < t reads both,
//            forms w_k = centred(u_k - v_k p^-1 mod q_t) and writes
//            out_k,i = (acc_k,i p^-1 - NTT_i(v_k p^-1 + w_k)) q_t^-1.
//
// This is, limb by limb, the same modular arithmetic as the three-kernel path
// (ctmul.cu; ModDown and rescale merged by linearity, limb t of the ModDown in
// the coefficient domain), so the outputs are bit-identical canonical
// residues.  Transforms per CTA: level + 2 for every CTA (5 at level 3), 20 in
// all at level 3, as in the three-kernel path.
//
// Barriers: every CTA executes the same six cluster barriers (split
// arrive / wait), unconditionally: no CTA leaves early, so none waits for one
// that never arrives, and none exits while another may still read its shared
// memory (the last wait follows the last remote read).
//
// Shared memory per CTA: the transform workspace, the published polynomial
// (N doubles) and the poly-1 accumulator (N doubles); the poly-0 accumulator
// lives in registers.  At N = 2^12: 98 KB, two CTAs of 256 threads per SM.
// Built for log N in [10, 13] with 16 coefficients per thread (radix-16
// register passes) and level in [2, 7] (clusters of at most 8 CTAs, the
// portable limit; the accumulators then stay below 11.5 q < 2^51 for
// q < 2^47 without folding).
#include <cooperative_groups.h>

#include <mutex>

#include "ctmul.hpp"
#include "dispatch.cuh"
#include "profile.hpp"
#include "tmem.cuh"

namespace cg = cooperative_groups;

namespace {

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// The same pointer, opaque to the compiler: the table loads of two transforms
// through two laundered copies are never merged (the loads are asm the
// compiler treats as pure), so no transform keeps another's twiddles live.
template <typename T>
__device__ __forceinline__ const T* opaque(const T* p) {
  const T* q;
  asm volatile("mov.b64 %0, %1;" : "=l"(q) : "l"(p));
  return q;
}
// The same shared-memory object of CTA `rank` of this cluster.
__device__ __forceinline__ const double* remote(double* local, unsigned rank) {
  return cg::this_cluster().map_shared_rank(local, rank);
}

constexpr int kFusedK = 4;         // coefficients per thread: 16
constexpr int kFusedMaxLevel = 7;  // cluster of level + 1 <= 8 CTAs

template <int LOGN>
struct FusedShape {
  using Sh = NttShape<LOGN, kFusedK>;
  static constexpr int MINB = Sh::T >= 512 ? 1 : 512 / Sh::T;  // 128 registers per thread
  static constexpr int SMEM_BYTES = (Sh::SMEM_WORDS + Sh::N) * 8;  // transform workspace + published poly
  // two accumulators of 16 doubles = 64 32-bit cells per thread
  static constexpr uint32_t TMEM_COLS = tmem_cols_for(Sh::T, 64);
};

}  // namespace

// Stage-C constants of one CTA, computed once into shared memory and read at
// each use (a copy held in registers across the transforms and barriers of
// stage C would not fit the 128-register budget).
struct StageCConsts {
  double ptw, ptq;    // p^-1 mod q_t and its quotient by q_t
  double pvw, pvq;    // p^-1 mod q_r and its quotient by q_r
  double ciw, ciq;    // q_t^-1 mod q_r and its quotient by q_r
  double tqd, tqinv;  // q_t, 1 / q_t
  u64 thalf;          // (q_t - 1) / 2
};

// Per-thread accumulator cells in TMEM: acc_k element e (a double, two 32-bit
// cells) at column 32 k + 2 e of the thread's 64-column range; moved in
// chunks of 8 elements.
__device__ __forceinline__ uint32_t acc_addr(uint32_t tbase, int k, int chunk) {
  return tbase + (uint32_t)(32 * k + 16 * chunk);
}

// Stage B tail: acc_k += x * key_k (x in layout C, key values natural order).
template <int LOGN>
__device__ __forceinline__ void key_product(const double (&x)[16], uint32_t tbase, const double* kp0,
                                            const double* kp1, int tid, const PrimeInfo& P) {
  constexpr int K = kFusedK;
#pragma unroll 1
  for (int k = 0; k < 2; ++k) {
    const double* kp = k ? kp1 : kp0;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      double w[8], a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) w[i] = ld_stream_d(kp + posC<LOGN, K>(tid, 8 * c + i));
      tmem_ld8(acc_addr(tbase, k, c), a);
#pragma unroll
      for (int i = 0; i < 8; ++i)
        a[i] = __dadd_rn(a[i], fmulmod(x[8 * c + i], w[i], __dmul_rn(w[i], P.qinv_d), P.qd));
      tmem_st8(acc_addr(tbase, k, c), a);
    }
  }
}

// Stage C producer: CTA p -> v_k = centred INTT_p(acc_k) (reduced first);
// CTA t -> u_k = INTT_t(acc_k p^-1).  Result in layout C in z.
template <int LOGN>
__device__ __forceinline__ void produce(double (&z)[16], int k, bool special, uint32_t tbase, u64* sm, int tid,
                                        const TwD* tb, const PrimeInfo& P, const StageCConsts& cc) {
  constexpr int K = kFusedK;
  double d[16];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    double a[8];
    tmem_ld8(acc_addr(tbase, k, c), a);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      d[8 * c + i] = special ? dreduce(a[i], P.qd, P.qinv_d) : fmulmod(a[i], cc.ptw, cc.ptq, P.qd);  // |.| <= q
  }
  c_to_z<LOGN, K>(d, sm, tid);
  u64 xo[16];
  ntt_inv_d<LOGN, K>(d, xo, sm, tid, opaque(tb), P);
#pragma unroll
  for (int e = 0; e < 16; ++e) z[e] = (special && xo[e] > P.half) ? __dadd_rn(u2d(xo[e]), -P.qd) : u2d(xo[e]);
}

// Stage C consumer, first half: the NTT input v p^-1 + w (|.| < 2 q_r), with
// w = centred(u - v p^-1 mod q_t), from the published v_k (CTA p) and u_k (CTA t).
template <int LOGN>
__device__ __forceinline__ void consume_prepare(double (&d)[16], const double* vp, const double* up, int tid,
                                                const PrimeInfo& P, const StageCConsts& cc) {
  constexpr int K = kFusedK;
  const double ptw = cc.ptw, ptq = cc.ptq, pvw = cc.pvw, pvq = cc.pvq;
  const double tqd = cc.tqd, tqinv = cc.tqinv;
  const u64 thalf = cc.thalf;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int pos = posC<LOGN, K>(tid, e);
    const double v = vp[pos];
    const u64 w = d2canon(__dadd_rn(up[pos], -fmulmod(v, ptw, ptq, tqd)), tqd, tqinv);
    const double wc = w > thalf ? __dadd_rn(u2d(w), -tqd) : u2d(w);
    d[e] = __dadd_rn(fmulmod(v, pvw, pvq, P.qd), wc);
  }
}

// Stage C consumer, second half: out_k,r = (acc_k p^-1 - NTT_r(d)) q_t^-1.
template <int LOGN>
__device__ __forceinline__ void consume_finish(double (&d)[16], int k, uint32_t tbase, u64* sm, int tid,
                                               const TwD* tb, const PrimeInfo& P, const StageCConsts& cc,
                                               u64* __restrict__ dst) {
  constexpr int K = kFusedK;
  ntt_fwd_d<LOGN, K>(d, sm, tid, opaque(tb), P);  // |d| < 2^51
  z_to_c<LOGN, K>(d, sm, tid);
  const double pvw = cc.pvw, pvq = cc.pvq, ciw = cc.ciw, ciq = cc.ciq;
  u64 o[16];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    double a[8];
    tmem_ld8(acc_addr(tbase, k, c), a);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double sd = __dadd_rn(fmulmod(a[i], pvw, pvq, P.qd), -d[8 * c + i]);
      o[8 * c + i] = d2canon(fmulmod(sd, ciw, ciq, P.qd), P.qd, P.qinv_d);
    }
  }
  store_c<LOGN, K>(o, dst, tid);
}

template <int LOGN>
__global__ void __launch_bounds__(NttShape<LOGN, kFusedK>::T, FusedShape<LOGN>::MINB)
    k_cm_fused(const u64* __restrict__ A, const u64* __restrict__ B, const double* __restrict__ key,
               u64* __restrict__ out, int level, int nq, const PrimeInfo* __restrict__ pi,
               const TwD* __restrict__ tw, const TwPair* __restrict__ pinv,
               const TwPair* __restrict__ qtinv) {
  constexpr int K = kFusedK;
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  constexpr int E = Sh::E;
  static_assert(E == 16, "the accumulator layout assumes 16 coefficients per thread");
  extern __shared__ __align__(16) u64 sm[];
  __shared__ uint32_t tmem_slot;
  __shared__ StageCConsts cc;
  double* pub = reinterpret_cast<double*>(sm + Sh::SMEM_WORDS);  // [N] published polynomial (layout C)

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int r = (int)cluster_rank();
  const int t = level - 1;
  const bool special = r == level;
  if (tid == 32) {
    // stage-C constants (CTAs r < t use all; CTA t uses ptw, ptq)
    const double tq = (double)pi[t].q;
    const double rq = (double)pi[special ? nq : r].q;
    cc.tqd = tq;
    cc.tqinv = pi[t].qinv_d;
    cc.thalf = pi[t].half;
    cc.ptw = (double)pinv[t].w;
    cc.ptq = __ddiv_rn(cc.ptw, tq);
    cc.pvw = special ? 0.0 : (double)pinv[r].w;
    cc.pvq = __ddiv_rn(cc.pvw, rq);
    cc.ciw = (special || r >= t) ? 0.0 : (double)qtinv[(size_t)t * nq + r].w;
    cc.ciq = __ddiv_rn(cc.ciw, rq);
  }
  // accumulators: 64 TMEM columns per thread (acc0 then acc1)
  if (warp == 0) tmem_alloc_warp(&tmem_slot, FusedShape<LOGN>::TMEM_COLS);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tbase = tmem_slot + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(64 * (tid >> 7));

  const int pidx = special ? nq : r;  // context prime index of this CTA's prime
  const long long ct = blockIdx.x / (level + 1);
  const PrimeInfo P = pi[pidx];
  const TwD* tb = twbase<LOGN>(tw, pidx);
  const size_t LN = (size_t)level * N;
  // key values of digit j, poly k, this CTA's prime (N doubles, natural order)
  const size_t kstride = (size_t)(nq + 1) * 2 * N;  // next poly k
  const double* key_r = key + (size_t)pidx * 2 * N;   // digit 0, poly 0, this prime

  // ------------------------------------------------------------ stage A
  if (!special) {
    const u64* a0 = A + ct * 2 * LN + (size_t)r * N;
    const u64* b0 = B + ct * 2 * LN + (size_t)r * N;
    const double pw = (double)(pi[nq].q % P.q);  // [p]_{q_r}
    const double pwq = __ddiv_rn(pw, P.qd);
    const double* k0 = key_r + (size_t)r * 2 * kstride;
    const double* k1 = k0 + kstride;
    double m2d[E];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      double c0[8], c1[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int e = 8 * c + i;
        const int pos = posC<LOGN, K>(tid, e);
        const double a0d = u2d(ld_stream(a0 + pos)), a1d = u2d(ld_stream(a0 + LN + pos));
        const double b0d = u2d(ld_stream(b0 + pos)), b1d = u2d(ld_stream(b0 + LN + pos));
        const double m2 = fmulmod_var(a1d, b1d, P.qd, P.qinv_d);  // |.| < q
        const double m0 = fmulmod_var(a0d, b0d, P.qd, P.qinv_d);
        const double s1 = fmulmod_var(__dadd_rn(a0d, a1d), __dadd_rn(b0d, b1d), P.qd, P.qinv_d);
        const double d1 = __dadd_rn(__dadd_rn(s1, -m0), -m2);     // |.| < 3 q
        const double w0 = ld_stream_d(k0 + pos), w1 = ld_stream_d(k1 + pos);
        c0[i] = __dadd_rn(fmulmod(m0, pw, pwq, P.qd), fmulmod(m2, w0, __dmul_rn(w0, P.qinv_d), P.qd));
        c1[i] = __dadd_rn(fmulmod(d1, pw, pwq, P.qd), fmulmod(m2, w1, __dmul_rn(w1, P.qinv_d), P.qd));
        m2d[e] = m2;
      }
      tmem_st8(acc_addr(tbase, 0, c), c0);
      tmem_st8(acc_addr(tbase, 1, c), c1);
    }
    // digit r: INTT_r(d2), canonical residues in [0, q_r), published
    u64 dg[E];
    c_to_z<LOGN, K>(m2d, sm, tid);  // |m2d| < q: straight into the FP64 inverse
    ntt_inv_d<LOGN, K>(m2d, dg, sm, tid, opaque(tb), P);
#pragma unroll
    for (int e = 0; e < E; ++e) pub[posC<LOGN, K>(tid, e)] = u2d(dg[e]);
  } else {
    const double zero[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int c = 0; c < 2; ++c) tmem_st8(acc_addr(tbase, k, c), zero);
  }
  cluster_arrive();  // B1: digits published
  cluster_wait();

  // ------------------------------------------------------------ stage B
#pragma unroll 1
  for (int j = 0; j < level; ++j) {
    if (j == r) continue;  // uniform across the CTA
    const double* src = remote(pub, (unsigned)j);
    double x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = src[posC<LOGN, K>(tid, e)];  // [0, q_j), < 2 q
    ntt_fwd_d<LOGN, K>(x, sm, tid, opaque(tb), P);                    // |x| < 2^51
    z_to_c<LOGN, K>(x, sm, tid);
    const double* k0 = key_r + (size_t)j * 2 * kstride;
    key_product<LOGN>(x, tbase, k0, k0 + kstride, tid, P);
  }
  cluster_arrive();  // B2: every remote digit read
  cluster_wait();

  // ------------------------------------------------------------ stage C
  if (special || r == t) {
    // producers: k = 0 -> B3 published, B4 consumed; k = 1 -> B5, B6
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
      double z[E];
      produce<LOGN>(z, k, special, tbase, sm, tid, tb, P, cc);
      if (k == 1) cluster_wait();  // B4: k = 0 consumed
#pragma unroll
      for (int e = 0; e < E; ++e) pub[posC<LOGN, K>(tid, e)] = z[e];
      cluster_arrive();  // B3 / B5: k published
      cluster_wait();
      cluster_arrive();  // B4 / B6
    }
    cluster_wait();  // B6: k = 1 consumed; the buffer may go
  } else {
    // consumers: output limb r of both polynomials
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
      double d[E];
      cluster_arrive();  // B3 / B5
      cluster_wait();    // k published
      consume_prepare<LOGN>(d, remote(pub, (unsigned)level), remote(pub, (unsigned)t), tid, P, cc);
      cluster_arrive();  // B4 / B6: k read
      consume_finish<LOGN>(d, k, tbase, sm, tid, tb, P, cc,
                           out + ((size_t)ct * 2 + k) * (size_t)t * N + (size_t)r * N);
      cluster_wait();
    }
  }
  // every TMEM access of every thread is complete (each helper waits for its own)
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc_warp(tmem_slot, FusedShape<LOGN>::TMEM_COLS);
}

namespace {

template <int LOGN>
cudaLaunchConfig_t fused_config(int n_ct, int level, int smem, cudaStream_t st, cudaLaunchAttribute* attr) {
  using Sh = NttShape<LOGN, kFusedK>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)((long long)n_ct * (level + 1)), 1, 1);
  cfg.blockDim = dim3(Sh::T, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = level + 1;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Per device and log N, looked up once: the dynamic shared memory each CTA
// requests (at least the kernel's need, raised until the CTAs that fit on one
// SM hold at most the SM's 512 TMEM columns, so no tcgen05.alloc ever waits
// for another CTA's columns), and per level whether the device schedules the
// cluster (cudaOccupancyMaxActiveClusters).
std::mutex g_fused_mu;
int g_fused_smem[14][128];                            // 0 unknown, -1 unusable
signed char g_fused_ok[14][kFusedMaxLevel + 1][128];  // 0 unknown, 1 yes, -1 no

template <int LOGN>
int fused_smem_locked(int dev) {
  int& sm_bytes = g_fused_smem[LOGN][dev];
  if (sm_bytes != 0) return sm_bytes;
  using Sh = NttShape<LOGN, kFusedK>;
  auto kern = k_cm_fused<LOGN>;
  // the opt-in limit covers static + dynamic shared memory of a CTA
  cudaFuncAttributes fa = {};
  sm_bytes = -1;
  if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) {
    (void)cudaGetLastError();
    return sm_bytes;
  }
  const int limit = smem_optin_limit() - (int)fa.sharedSizeBytes;
  int bytes = FusedShape<LOGN>::SMEM_BYTES;
  const int max_ctas = 512 / (int)FusedShape<LOGN>::TMEM_COLS;
  if (bytes > limit || cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, limit) != cudaSuccess) {
    (void)cudaGetLastError();
    return sm_bytes;
  }
  for (; bytes <= limit; bytes += 1024) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Sh::T, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      return sm_bytes;
    }
    if (per_sm >= 1 && per_sm <= max_ctas) {
      sm_bytes = bytes;
      break;
    }
  }
  return sm_bytes;
}

template <int LOGN>
int fused_schedulable(int level) {  // dynamic smem bytes, or 0 when not schedulable
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) {
    (void)cudaGetLastError();
    return 0;
  }
  std::lock_guard<std::mutex> lk(g_fused_mu);
  const int smem = fused_smem_locked<LOGN>(dev);
  if (smem <= 0) return 0;
  signed char& ok = g_fused_ok[LOGN][level][dev];
  if (ok == 0) {
    int clusters = 0;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = fused_config<LOGN>(1, level, smem, nullptr, attr);
    if (cudaOccupancyMaxActiveClusters(&clusters, k_cm_fused<LOGN>, &cfg) != cudaSuccess) {
      (void)cudaGetLastError();
      clusters = 0;
    }
    ok = clusters > 0 ? 1 : -1;
  }
  return ok > 0 ? smem : 0;
}

template <int LOGN>
int fused_launch(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a, const uint64_t* ct_b,
                 const uint64_t* key, int n_ct, int level, cudaStream_t st, const char* fn) {
  const int smem = fused_schedulable<LOGN>(level);
  if (smem <= 0) return CKKS_EUNSUPPORTED;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = fused_config<LOGN>(n_ct, level, smem, st, attr);
  ProfSpan span(CKKS_STAGE_CM_FUSED, st);
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_cm_fused<LOGN>, reinterpret_cast<const u64*>(ct_a),
                                     reinterpret_cast<const u64*>(ct_b), reinterpret_cast<const double*>(key),
                                     reinterpret_cast<u64*>(out), level, ctx->n_q, (const PrimeInfo*)ctx->d_pi,
                                     (const TwD*)ctx->d_tw, (const TwPair*)ctx->d_pinv,
                                     (const TwPair*)ctx->d_qtinv);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: fused launch: %s", fn, cudaGetErrorString(e));
  return CKKS_OK;
}

}  // namespace

bool ckks_ct_mul_fused_supported(const ckks_ctx* ctx, int level) {
  return ctx->log_n >= 10 && ctx->log_n <= 13 && level >= 2 && level <= kFusedMaxLevel &&
         ctx->n_special == 1;
}

bool ckks_ct_mul_fused_will_run(const ckks_ctx* ctx, int level) {
  // opt-in (CKKS_TUNE_CM_FUSED = 1): measured slower than the three kernels at
  // every built shape on B200 (0.50-0.77x at N = 2^12, 2^13, level 2..7; its
  // CTAs idle at the cluster barriers while the special-prime CTA, which has
  // no tensor work and one transform more, catches up)
  if (ctx->tune_cm_fused != 1 || !ckks_ct_mul_fused_supported(ctx, level)) return false;
  switch (ctx->log_n) {
    case 10: return fused_schedulable<10>(level) > 0;
    case 11: return fused_schedulable<11>(level) > 0;
    case 12: return fused_schedulable<12>(level) > 0;
    default: return fused_schedulable<13>(level) > 0;
  }
}

int ckks_ct_mul_fused(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a, const uint64_t* ct_b,
                      const uint64_t* key, int n_ct, int level, void* stream, const char* fn) {
  if (!ckks_ct_mul_fused_supported(ctx, level)) return CKKS_EUNSUPPORTED;
  if (n_ct == 0) return CKKS_OK;
  cudaStream_t st = as_stream(stream);
  switch (ctx->log_n) {
    case 10: return fused_launch<10>(ctx, out, ct_a, ct_b, key, n_ct, level, st, fn);
    case 11: return fused_launch<11>(ctx, out, ct_a, ct_b, key, n_ct, level, st, fn);
    case 12: return fused_launch<12>(ctx, out, ct_a, ct_b, key, n_ct, level, st, fn);
    default: return fused_launch<13>(ctx, out, ct_a, ct_b, key, n_ct, level, st, fn);
  }
}
