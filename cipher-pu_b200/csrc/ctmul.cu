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
//                          (digit j at its own prime reuses the NTT-domain d2).
//   C  moddown+rescale (ct, k):
//                          v = centred(INTT_p(acc_k,p))        (coefficient)
//                          limb t : w = centred(INTT_t(d_k,t + acc_k,t p^-1)
//                                               - [v]_t p^-1)
//                          limb i<t: out = (d_k,i + acc_k,i p^-1
//                                           - NTT_i([v]_i p^-1 + [w]_i)) q_t^-1
//                          (ModDown and rescale conversions merged into one
//                          NTT per limb, and limb t's ModDown done in the
//                          coefficient domain, by linearity of the NTT;
//                          bit-identical to doing them one after the other).
// Transforms per ct-mult at level L: L + (L-1)L + L + 2(L + 1) = 20 at L = 3
// (vs 26 for the unmerged sequence).
//
// Arithmetic: exact FP64 on integer-valued doubles in all three kernels
// (transforms, products, key inner product, basis conversions); residues go
// back to canonical uint64 only where they are stored.
//
// Launch shape: K = log2 coefficients per thread (2..5: N/2^K threads,
// radix-2^K register passes), MINB = CTAs per SM the register budget is cut
// for (__launch_bounds__), work units per CTA, and the tensor kernel's form
// (one CTA per unit, or persistent and TMA-fed) are context tuning
// parameters.
#include <mutex>

#include "ctmul.hpp"
#include "ctmul_modup_tm.cuh"
#include "ctmul_units.cuh"
#include "dispatch.cuh"
#include "profile.hpp"

// Per-device streams and events for concurrent sub-batches (created on first
// use, kept for the life of the process).  The mutex serialises the
// fork / launch / join enqueue of calls from different host threads, which
// share these events.
namespace {
constexpr int kMaxSplit = 4;     // internal streams per device
constexpr int kMaxSub = 4;       // default sub-batches per call at most
constexpr int kPairsPerSub = 64; // default pairs per sub-batch
constexpr int kSplitDevices = 128;
struct SplitStreams {
  bool ready = false;
  std::mutex mu;
  cudaStream_t s[kMaxSplit];
  cudaEvent_t fork, join[kMaxSplit];
};
std::mutex g_split_init_mu;
SplitStreams g_split[kSplitDevices];

int split_streams_for_device(SplitStreams** out, const char* fn) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  if (dev < 0 || dev >= kSplitDevices)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: device %d beyond %d", fn, dev, kSplitDevices);
  std::lock_guard<std::mutex> lock(g_split_init_mu);
  SplitStreams& ss = g_split[dev];
  if (!ss.ready) {
    for (int i = 0; i < kMaxSplit && e == cudaSuccess; ++i) e = cudaStreamCreateWithFlags(&ss.s[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming);
    for (int i = 0; i < kMaxSplit && e == cudaSuccess; ++i)
      e = cudaEventCreateWithFlags(&ss.join[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    ss.ready = true;
  }
  *out = &ss;
  return CKKS_OK;
}
}  // namespace


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

// CTAs per SM that the register budget of a launch shape targets: "balanced"
// gives every thread 128 registers (max(1, 512 / T) CTAs of T threads; 255
// registers for K = 5, whose 32 values per thread spill at 128), "tight" 64
// (twice the CTAs; not built for 1024-thread CTAs).
template <int LOGN, int K, bool TIGHT>
struct CmBlocks {
  static constexpr int T = (1 << LOGN) >> K;
  static constexpr int THR = K >= 5 ? 256 : 512;  // resident threads per SM of the balanced budget
  static constexpr int B = T >= THR ? 1 : THR / T;
  static constexpr int value = (TIGHT && T < 1024) ? 2 * B : B;
};

// ct-mult kernels are instantiated for log N in [6, 14] with K in {3, 4}
// (K = 3 needs N / 8 <= 1024 threads) and both register budgets, for log N
// in [10, 12] with K = 2 (both budgets) and for log N in [10, 14] with K = 5
// (balanced only: 32 values per thread do not fit 64 registers).  N = 2^14
// needs more shared memory per CTA than B200 offers (the launch paths check
// and refuse it with a message).  Defaults: K = 4 for log N >= 10 (3 below),
// balanced budget: measured fastest at N = 2^12 (2 CTAs of 256 threads per
// SM) and 2^13 (1 CTA of 512).
// f is called as f.template operator()<L, K, MINB>().
template <typename F>
static int dispatch_cm(int log_n, int kreq, int mreq, F&& f, const char* fn) {
  const int k = kreq ? kreq : (log_n >= 10 ? 4 : 3);
  const int budget = mreq ? mreq : 1;
  if (k < 2 || k > 5) return ckks_set_error(CKKS_EUNSUPPORTED, "%s: K=%d not built", fn, k);
  if (budget != 1 && budget != 2)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: register budget %d not in {1, 2}", fn, budget);
  if (log_n < 6 || log_n > 14)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: log_n=%d outside [6, 14]", fn, log_n);
  if (((1 << log_n) >> k) > 1024)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: K=%d gives more than 1024 threads at log_n=%d",
                          fn, k, log_n);
  if ((k == 2 && (log_n < 10 || log_n > 12)) || (k == 5 && log_n < 10))
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: K=%d not built at log_n=%d", fn, k, log_n);
  if (k == 5 && budget == 2)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: K=5 is built with the balanced budget only", fn);
  const bool tight = budget == 2;
  auto go = [&]<int L>() -> int {
    if constexpr (L < 6) {
      return ckks_set_error(CKKS_EUNSUPPORTED, "%s: log_n=%d outside [6, 14]", fn, log_n);
    } else {
      if (k == 2) {
        if constexpr (L >= 10 && L <= 12) {
          return tight ? f.template operator()<L, 2, CmBlocks<L, 2, true>::value>()
                       : f.template operator()<L, 2, CmBlocks<L, 2, false>::value>();
        }
      } else if (k == 3) {
        if constexpr (((1 << L) >> 3) <= 1024) {
          return tight ? f.template operator()<L, 3, CmBlocks<L, 3, true>::value>()
                       : f.template operator()<L, 3, CmBlocks<L, 3, false>::value>();
        }
      } else if (k == 5) {
        if constexpr (L >= 10) {
          return f.template operator()<L, 5, CmBlocks<L, 5, false>::value>();
        }
      } else {
        return tight ? f.template operator()<L, 4, CmBlocks<L, 4, true>::value>()
                     : f.template operator()<L, 4, CmBlocks<L, 4, false>::value>();
      }
      return ckks_set_error(CKKS_EUNSUPPORTED, "%s: K=%d not built at log_n=%d", fn, k, log_n);
    }
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

// ---------------------------------------------------------------- kernel A
// One CTA per (ct, limb j) (body: cm_tensor_unit, ctmul_units.cuh).
template <int LOGN, int K, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, MINB)
    k_cm_tensor(const u64* __restrict__ A, const u64* __restrict__ B, CmScratch S, int level,
                const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw, int n_ct,
                long long n_units, int upc) {
  extern __shared__ u64 sm[];
  // `upc` work units per CTA, consecutive in the unit order
  for (int r = 0; r < upc; ++r) {
    const long long unit = (long long)blockIdx.x * upc + r;
    if (unit >= n_units) return;  // uniform across the CTA
    if (r) __syncthreads();       // the previous unit is done with shared memory
    cm_tensor_unit<LOGN, K>(A, B, S, level, pi, tw, n_ct, unit, sm, threadIdx.x);
  }
}

// The tensor kernel the ct-mult uses unless CKKS_TUNE_CM_TENSOR_TMA says
// otherwise: one CTA per unit, measured faster than the TMA-fed persistent
// variant at N = 2^12, L = 3, 256 pairs (0.050 against 0.054 ms): the kernel
// is bound by its issue rate at 16 warps per SM more than by load latency,
// and the staged variant adds two barriers per quarter.
constexpr bool kTensorTmaDefault = false;

// ---------------------------------------------------------------- kernel A, TMA-fed
// Persistent variant of kernel A: each CTA walks the units blockIdx.x,
// blockIdx.x + gridDim.x, ...  The four input limbs of a unit arrive in
// quarters (N / 4 coefficients of a0, a1, b0, b1 per quarter) by bulk
// asynchronous copies into two shared-memory stages, each completing on its
// own mbarrier; one thread issues the copy of the quarter after next as soon
// as the CTA has read a stage, so the loads of quarters 2-3 and of the next
// unit's quarters 0-1 run under the products and the INTT of the current
// unit.  Every wait is bounded by `wait_limit` SM cycles (context tuning
// CKKS_TUNE_WAIT_CYCLES, default about 1 s): on expiry the CTA counts the
// event in g_cm_wait_expiries (read by ckks_device_status), thread 0 waits
// (bounded again, kDrainCycles) for every copy it issued that has not been
// waited for, so nothing is still landing in shared memory, and the CTA stops.
namespace {
__device__ unsigned int g_cm_wait_expiries;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of the given parity to complete; false after `limit` SM
// cycles without it.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test(bar, parity)) {
    if (clock64() - t0 > limit) return false;
    __nanosleep(20);
  }
  return true;
}
// Limit of the drain that follows an expired wait: the copies still in flight
// into the CTA's shared memory must land before the CTA may exit (about 2 s).
constexpr long long kDrainCycles = 4000000000ll;

// Shared memory of the TMA-fed tensor kernel: the transform workspace, two
// stages of 4 quarter-limbs, two mbarriers.
template <int LOGN, int K>
constexpr int tensor_tma_smem_bytes() {
  using Sh = NttShape<LOGN, K>;
  return (((Sh::SMEM_WORDS + 15) & ~15) + 2 * Sh::N) * 8 + 16;
}

template <int LOGN, int K, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, MINB)
    k_cm_tensor_tma(const u64* __restrict__ A, const u64* __restrict__ B, CmScratch S, int level,
                    const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw, int n_ct,
                    long long n_units, long long wait_limit) {
  extern __shared__ __align__(128) u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  constexpr int T = Sh::T;
  constexpr int QN = N / 4;         // coefficients per quarter
  constexpr int QE = Sh::E / 4;     // values a thread holds per quarter
  static_assert(Sh::E >= 4, "quarters need at least 4 values a thread");
  u64* stage[2];
  stage[0] = sm + ((Sh::SMEM_WORDS + 15) & ~15);
  stage[1] = stage[0] + 4 * QN;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(stage[1] + 4 * QN);
  const uint32_t bar[2] = {smem_u32(&bars[0]), smem_u32(&bars[1])};
  const int tid = threadIdx.x;
  const size_t LN = (size_t)level * N;
  if (tid == 0) {
    mbar_init(bar[0], 1);
    mbar_init(bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // copies issued into / completions waited for on each stage; the k-th
  // completion of a stage's barrier has parity k & 1 (issued: thread 0 only)
  int n_issued[2] = {0, 0}, n_waited[2] = {0, 0};
  // quarter q (a0, a1, b0, b1) of unit u into stage s
  auto issue = [&](long long u, int q, int s) {
    ++n_issued[s];
    const int j = (int)(u / n_ct);
    const long long ct = u % n_ct;
    const u64* a0 = A + ct * 2 * LN + (size_t)j * N + (size_t)q * QN;
    const u64* b0 = B + ct * 2 * LN + (size_t)j * N + (size_t)q * QN;
    mbar_expect_tx(bar[s], 4 * QN * 8);
    bulk_g2s(smem_u32(stage[s]), a0, QN * 8, bar[s]);
    bulk_g2s(smem_u32(stage[s] + QN), a0 + LN, QN * 8, bar[s]);
    bulk_g2s(smem_u32(stage[s] + 2 * QN), b0, QN * 8, bar[s]);
    bulk_g2s(smem_u32(stage[s] + 3 * QN), b0 + LN, QN * 8, bar[s]);
  };
  if (tid == 0 && (long long)blockIdx.x < n_units) {
    issue(blockIdx.x, 0, 0);
    issue(blockIdx.x, 1, 1);
  }
  bool expired = false;
  for (long long u = blockIdx.x; u < n_units && !expired; u += gridDim.x) {
    const int j = (int)(u / n_ct);
    const long long ct = u % n_ct;
    const PrimeInfo P = pi[j];
    u64* d0 = S.d01 + ct * 2 * LN + (size_t)j * N;
    u64* d2n = S.d2n + ct * LN + (size_t)j * N;
    const long long un = u + gridDim.x;
    double m2d[Sh::E];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int s = q & 1;
      const bool ok = mbar_wait(bar[s], n_waited[s] & 1, wait_limit);
      if (__syncthreads_or(!ok)) {
        expired = true;
        break;
      }
      ++n_waited[s];
      const u64* st = stage[s];
      // FP64 products as in kernel A; this thread's values of the quarter
      // are positions q N/4 + tid + T e2 (layout C)
#pragma unroll
      for (int e2 = 0; e2 < QE; ++e2) {
        const int l = tid + T * e2;
        const int pos = q * QN + l;
        const double a0d = u2d(st[l]), a1d = u2d(st[QN + l]);
        const double b0d = u2d(st[2 * QN + l]), b1d = u2d(st[3 * QN + l]);
        const double m2 = fmulmod_var(a1d, b1d, P.qd, P.qinv_d);
        const double m0 = fmulmod_var(a0d, b0d, P.qd, P.qinv_d);
        const double s1 = fmulmod_var(__dadd_rn(a0d, a1d), __dadd_rn(b0d, b1d), P.qd, P.qinv_d);
        d0[pos] = d2canon(m0, P.qd, P.qinv_d);
        d0[LN + pos] = d2canon(__dadd_rn(__dadd_rn(s1, -m0), -m2), P.qd, P.qinv_d);
        d2n[pos] = d2canon(m2, P.qd, P.qinv_d);
        m2d[q * QE + e2] = m2;
      }
      __syncthreads();  // the stage has been read by every thread
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (q < 2)
          issue(u, q + 2, s);
        else if (un < n_units)
          issue(un, q - 2, s);
      }
    }
    if (expired) break;
    u64 m2[Sh::E];
    c_to_z<LOGN, K>(m2d, sm, tid);  // |m2d| < 0.6 q: straight into the FP64 inverse
    ntt_inv_d<LOGN, K>(m2d, m2, sm, tid, twbase<LOGN>(tw, j), P);
    store_c<LOGN, K>(m2, S.d2c + ct * LN + (size_t)j * N, tid);
  }
  if (expired && tid == 0) {
    atomicAdd(&g_cm_wait_expiries, 1u);
    for (int st = 0; st < 2; ++st)
      for (; n_waited[st] < n_issued[st]; ++n_waited[st])
        if (!mbar_wait(bar[st], n_waited[st] & 1, kDrainCycles)) {
          atomicAdd(&g_cm_wait_expiries, 1u);  // still in flight after the drain limit
          break;
        }
  }
  __syncthreads();  // no thread leaves before the drain
}

// expiries of the tensor-core linear layer's waits (linear_tc.cu), read and cleared
int ckks_linear_tc_status_take(unsigned int* n);
int ckks_batch_status_take(unsigned int* n);
int ckks_ntt_tc_status_take(unsigned int* n);

extern "C" int ckks_device_status(void) {
  unsigned int n = 0, n_tc = 0, n_pb = 0, n_nt = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&n, g_cm_wait_expiries, sizeof(n));
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  if (n) {
    const unsigned int zero = 0;
    e = cudaMemcpyToSymbol(g_cm_wait_expiries, &zero, sizeof(zero));
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  }
  if (int rc = ckks_linear_tc_status_take(&n_tc)) return rc;
  if (int rc = ckks_batch_status_take(&n_pb)) return rc;
  if (int rc = ckks_ntt_tc_status_take(&n_nt)) return rc;
  const unsigned int total = n + n_tc + n_pb + n_nt;
  if (total == 0) return CKKS_OK;
  return ckks_set_error(CKKS_ETIMEOUT, "ckks_device_status: %u bounded device waits expired", total);
}

// ---------------------------------------------------------------- kernel B
// One CTA per (ct, target prime).  Each digit is transformed (layout C in,
// Z out) and re-distributed to layout C, so the key limbs, stored in natural
// order, are read lane-contiguously.  The two accumulators live in
// thread-private shared-memory slots (index e * T + tid).
template <int LOGN, int K, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, MINB)
    k_cm_modup(CmScratch S, const double* __restrict__ key, int level, int nq,
               const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw, int n_ct,
                long long n_units, int upc) {
  extern __shared__ u64 sm[];
  // `upc` work units per CTA, consecutive in the unit order (body: cm_modup_unit)
  for (int r = 0; r < upc; ++r) {
    const long long unit = (long long)blockIdx.x * upc + r;
    if (unit >= n_units) return;  // uniform across the CTA
    if (r) __syncthreads();       // the previous unit is done with shared memory
    cm_modup_unit<LOGN, K, false>(S, key, level, nq, pi, tw, n_ct, unit, sm, threadIdx.x);
  }
}

// ---------------------------------------------------------------- kernel C
// One CTA per (ct, poly k), all in FP64 on exact doubles: the special-prime
// part v and the rescale limb w are kept centred (signed, |v| <= p / 2,
// |w| <= q_t / 2) in thread-private shared-memory slots (layout C), so they
// lift to any prime as they are.  Products by p^-1 and q_t^-1 are fmulmod
// with w / q correctly rounded (|result| <= q).  Bounds: the forward
// transform gets |x| < 2 q_i (q_t < 2 q_i) and returns |x| < 13.75 q; the
// combination stays below 16 q < 2^51; the inverses get |x| <= 1.5 q.
template <int LOGN, int K, int MINB, bool MULTI>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, MINB)
    k_cm_down(CmScratch S, u64* __restrict__ out, int level, int nq,
              const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw,
              const TwPair* __restrict__ pinv, const TwPair* __restrict__ qtinv, long long n_units,
              int upc) {
  extern __shared__ u64 sm[];
  // `upc` work units per CTA, consecutive in the unit order (body: cm_down_unit)
  for (int r = 0; r < (MULTI ? upc : 1); ++r) {
    const long long unit = (long long)blockIdx.x * upc + r;
    if (MULTI && unit >= n_units) return;  // uniform across the CTA
    if (r) __syncthreads();       // the previous unit is done with shared memory
    cm_down_unit<LOGN, K, false>(S, out, level, nq, pi, tw, pinv, qtinv, unit, sm, threadIdx.x);
  }
}

// ---------------------------------------------------------------- rotation
// Galois key switch of psi_nu(ct) (ckks_rotate): kernel R1 permutes both
// polynomials in the evaluation domain (psi(c0) -> d01 slot 0, psi(c1) ->
// d2n, and its INTT -> d2c, the digits), kernel B above forms the key inner
// product with the Galois key, kernel R3 divides by the special prime
// (ModDown, no rescale) and adds psi(c0).
template <int LOGN, int K, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, MINB)
    k_rot_prep(const u64* __restrict__ C, CmScratch S, int level, u64 nu2n,
               const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw, int n_ct,
                long long n_units, int upc) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  // `upc` work units per CTA, consecutive in the unit order
  for (int r = 0; r < upc; ++r) {
    const long long unit = (long long)blockIdx.x * upc + r;
    if (unit >= n_units) return;  // uniform across the CTA
    if (r) __syncthreads();       // the previous unit is done with shared memory
    const int j = unit / n_ct;
    const long long ct = unit % n_ct;
    const int tid = threadIdx.x;
    const PrimeInfo P = pi[j];
    const size_t LN = (size_t)level * N;
    const u64* c0 = C + ct * 2 * LN + (size_t)j * N;
    u64 x[Sh::E];
  #pragma unroll
    for (int e = 0; e < Sh::E; ++e) x[e] = ld_stream(c0 + galois_eval_src(posC<LOGN, K>(tid, e), LOGN, nu2n));
    store_c<LOGN, K>(x, S.d01 + ct * 2 * LN + (size_t)j * N, tid);
  #pragma unroll
    for (int e = 0; e < Sh::E; ++e)
      x[e] = ld_stream(c0 + LN + galois_eval_src(posC<LOGN, K>(tid, e), LOGN, nu2n));
    store_c<LOGN, K>(x, S.d2n + ct * LN + (size_t)j * N, tid);
    c_to_z<LOGN, K>(x, sm, tid);
    ntt_inv<LOGN, K>(x, sm, tid, twbase<LOGN>(tw, j), P);
    store_c<LOGN, K>(x, S.d2c + ct * LN + (size_t)j * N, tid);
  }
}

// kernel R3: one CTA per (ct, poly k): v = centred INTT_p(acc_k,p); every
// limb i: out_k,i = [k == 0] psi(c0)_i + (acc_k,i - NTT_i(v)) p^-1, in FP64
// like kernel C (v kept signed in shared memory; |v| < q_i since p < 2 q_i).
template <int LOGN, int K, int MINB, bool MULTI>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T, MINB)
    k_ks_down(CmScratch S, u64* __restrict__ out, int level, int nq, const PrimeInfo* __restrict__ pi,
              const TwD* __restrict__ tw, const TwPair* __restrict__ pinv, long long n_units,
              int upc) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  constexpr int T = Sh::T;
  double* vs = reinterpret_cast<double*>(sm + Sh::SMEM_WORDS);
  // `upc` work units per CTA, consecutive in the unit order
  for (int r = 0; r < (MULTI ? upc : 1); ++r) {
    const long long unit = (long long)blockIdx.x * upc + r;
    if (MULTI && unit >= n_units) return;  // uniform across the CTA
    if (r) __syncthreads();       // the previous unit is done with shared memory
    const long long ct = unit >> 1;
    const int k = unit & 1;
    const int tid = threadIdx.x;
    const size_t LN = (size_t)level * N;
    const PrimeInfo PP = pi[nq];
    const u64* d0 = S.d01 + ct * 2 * LN;
    const u64* ak = S.acc + ct * 2 * LN + (size_t)k * LN;
    u64* ok = out + ((size_t)ct * 2 + k) * LN;
    double d[Sh::E];
    u64 x[Sh::E];
    load_c<LOGN, K>(x, S.accp + (ct * 2 + k) * N, tid);
  #pragma unroll
    for (int e = 0; e < Sh::E; ++e) d[e] = u2d(x[e]);
    c_to_z<LOGN, K>(d, sm, tid);
    ntt_inv_d<LOGN, K>(d, x, sm, tid, twbase<LOGN>(tw, nq), PP);
  #pragma unroll
    for (int e = 0; e < Sh::E; ++e) vs[e * T + tid] = x[e] > PP.half ? u2d(x[e]) - PP.qd : u2d(x[e]);
  #pragma unroll 1
    for (int i = 0; i < level; ++i) {
      const PrimeInfo P = pi[i];
      const double pvw = (double)pinv[i].w;
      const double pvq = __ddiv_rn(pvw, P.qd);
  #pragma unroll
      for (int e = 0; e < Sh::E; ++e) d[e] = vs[e * T + tid];
      ntt_fwd_d<LOGN, K>(d, sm, tid, twbase<LOGN>(tw, i), P);  // |d| < 13.75 q
      z_to_c<LOGN, K>(d, sm, tid);
      u64 av[Sh::E];
      load_c<LOGN, K>(av, ak + (size_t)i * N, tid);
  #pragma unroll
      for (int e = 0; e < Sh::E; ++e) d[e] = fmulmod(__dadd_rn(u2d(av[e]), -d[e]), pvw, pvq, P.qd);
      if (k == 0) {
        load_c<LOGN, K>(av, d0 + (size_t)i * N, tid);
  #pragma unroll
        for (int e = 0; e < Sh::E; ++e) d[e] = __dadd_rn(d[e], u2d(av[e]));
      }
  #pragma unroll
      for (int e = 0; e < Sh::E; ++e) x[e] = d2canon(d[e], P.qd, P.qinv_d);
      store_c<LOGN, K>(x, ok + (size_t)i * N, tid);
    }
  }
}

// ---------------------------------------------------------------- key prep
// Prepared key: per (digit, poly, limb) a block of 2N doubles, the N values w
// followed by their N quotients w / q (the ModUp kernel streams only the
// values and forms w / q itself; the quotients serve callers that want both).
__global__ void k_key_prepare(double* __restrict__ out, const u64* __restrict__ in,
                              long long total, int log_n, int nlimb,
                              const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const long long blk = idx >> log_n;
  const long long i = idx & ((1ll << log_n) - 1);
  const PrimeInfo P = pi[(int)(blk % nlimb)];
  const double w = u2d(in[idx] % P.q);
  out[(blk << (log_n + 1)) + i] = w;
  out[(blk << (log_n + 1)) + (1ll << log_n) + i] = __ddiv_rn(w, P.qd);
}

extern "C" int ckks_relin_key_prepare(const ckks_ctx* ctx, uint64_t* prepared,
                                      const uint64_t* ksk, void* stream) {
  CKKS_REQUIRE(ctx != nullptr, "ckks_relin_key_prepare: ctx is NULL");
  CKKS_REQUIRE(ctx->n_special == 1, "ckks_relin_key_prepare: context needs one special prime");
  const long long total = (long long)ctx->n_q * 2 * ctx->n_primes * ctx->n;
  k_key_prepare<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<double*>(prepared), reinterpret_cast<const u64*>(ksk), total,
      ctx->log_n, ctx->n_primes, ctx->d_pi);
  return ckks_check_launch("ckks_relin_key_prepare");
}

size_t ckks_ct_mul_scratch_bytes_3k(const ckks_ctx* ctx, int n_ct, int level) {
  if (!ctx || n_ct < 0 || level < 1) return 0;
  return cm_words(ctx->n, n_ct, level) * sizeof(u64);
}

extern "C" size_t ckks_ct_mul_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level) {
  if (!ctx || n_ct < 0 || level < 1) return 0;
  if (ckks_ct_mul_fused_will_run(ctx, level)) return 0;
  return ckks_ct_mul_scratch_bytes_3k(ctx, n_ct, level);
}

// The three ct-mult kernels for one sub-batch on one stream.
static int cm_launch_one(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a, const uint64_t* ct_b,
                         const uint64_t* key, int n_ct, int level, CmScratch S, cudaStream_t st,
                         const char* fn) {
  return dispatch_cm(ctx->log_n, ctx->tune_cm_k, ctx->tune_cm_minb, [&]<int L, int K, int MINB>() -> int {
    using Sh = NttShape<L, K>;
    const int upc = ctx->tune_cm_upc ? ctx->tune_cm_upc : 1;
    const int smem_a = Sh::SMEM_WORDS * 8;
    const int smem_bc = (Sh::SMEM_WORDS + 2 * Sh::N) * 8;
    if (int rc = require_smem(smem_bc, L, fn)) return rc;
    auto ka = k_cm_tensor<L, K, MINB>;
    auto kb = k_cm_modup<L, K, MINB>;
    // one unit per CTA builds without the unit loop (it costs ModDown registers)
    auto kc = upc > 1 ? k_cm_down<L, K, MINB, true> : k_cm_down<L, K, MINB, false>;
    ensure_smem(ka, smem_a);
    ensure_smem(kb, smem_bc);
    ensure_smem(kc, smem_bc);
    if (ctx->tune_cm_tma == 1 || (ctx->tune_cm_tma == 0 && kTensorTmaDefault)) {
      // persistent, TMA-fed: as many CTAs as fit at once, each walking units
      CKKS_REQUIRE(((reinterpret_cast<uintptr_t>(ct_a) | reinterpret_cast<uintptr_t>(ct_b)) & 15) == 0,
                   "%s: the TMA-fed tensor kernel needs 16-byte aligned inputs", fn);
      auto kt = k_cm_tensor_tma<L, K, MINB>;
      const int smem_t = tensor_tma_smem_bytes<L, K>();
      if (int rc = require_smem(smem_t, L, fn)) return rc;
      ensure_smem(kt, smem_t);
      int dev = 0, n_sm = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kt, Sh::T, smem_t);
      const long long nu_a = (long long)n_ct * level;
      long long grid = (long long)(n_sm > 0 ? n_sm : 1) * (per_sm > 0 ? per_sm : 1);
      grid = grid < nu_a ? grid : nu_a;
      ProfSpan span(CKKS_STAGE_CM_TENSOR, st);
      kt<<<grid1d(grid), Sh::T, smem_t, st>>>(reinterpret_cast<const u64*>(ct_a),
                                               reinterpret_cast<const u64*>(ct_b), S, level, ctx->d_pi,
                                               ctx->d_tw, n_ct, nu_a, ckks_wait_limit(ctx));
    } else {
      ProfSpan span(CKKS_STAGE_CM_TENSOR, st);
      const long long nu_a = (long long)n_ct * level;
      ka<<<grid1d((nu_a + upc - 1) / upc), Sh::T, smem_a, st>>>(
          reinterpret_cast<const u64*>(ct_a), reinterpret_cast<const u64*>(ct_b), S, level,
          ctx->d_pi, ctx->d_tw, n_ct, nu_a, upc);
    }
    if (int rc = ckks_check_launch(fn)) return rc;
    {
      ProfSpan span(CKKS_STAGE_CM_MODUP, st);
      const long long nu_b = (long long)n_ct * (level + 1);
      bool tm = false;
      if constexpr (ModupTm<L, K>::BUILT) {
        if (ctx->tune_cm_tmem != 2) {
          // accumulators in TMEM: the CTA needs only its transform buffer
          k_cm_modup_tm<L, K><<<grid1d((nu_b + upc - 1) / upc), Sh::T, smem_a, st>>>(
              S, reinterpret_cast<const double*>(key), level, ctx->n_q, ctx->d_pi, ctx->d_tw, n_ct, nu_b, upc);
          tm = true;
        }
      }
      if (!tm)
        kb<<<grid1d((nu_b + upc - 1) / upc), Sh::T, smem_bc, st>>>(
            S, reinterpret_cast<const double*>(key), level, ctx->n_q, ctx->d_pi, ctx->d_tw, n_ct, nu_b, upc);
    }
    if (int rc = ckks_check_launch(fn)) return rc;
    {
      ProfSpan span(CKKS_STAGE_CM_DOWN, st);
      const long long nu_c = (long long)n_ct * 2;
      kc<<<grid1d((nu_c + upc - 1) / upc), Sh::T, smem_bc, st>>>(
          S, reinterpret_cast<u64*>(out), level, ctx->n_q, ctx->d_pi, ctx->d_tw, ctx->d_pinv,
          ctx->d_qtinv, nu_c, upc);
    }
    return ckks_check_launch(fn);
  }, fn);
}

int ckks_ct_mul_launch(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                       const uint64_t* ct_b, const uint64_t* key, int n_ct, int level,
                       void* scratch, size_t scratch_bytes, void* stream, const char* fn,
                       int max_split, bool allow_fused) {
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(ctx->n_special == 1, "%s: context needs exactly one special prime", fn);
  CKKS_REQUIRE(level >= 2 && level <= ctx->n_q, "%s: level=%d outside [2, %d]", fn, level,
               ctx->n_q);
  CKKS_REQUIRE(ctx->log_n >= 6, "%s: log_n=%d below the supported minimum 6", fn, ctx->log_n);
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
  if (allow_fused && ckks_ct_mul_fused_will_run(ctx, level)) {
    CKKS_REQUIRE(out && ct_a && ct_b && key, "%s: NULL pointer argument", fn);
    const int rc = ckks_ct_mul_fused(ctx, out, ct_a, ct_b, key, n_ct, level, stream, fn);
    if (rc != CKKS_EUNSUPPORTED) return rc;
  }
  if (allow_fused && ctx->tune_cm_fused == 1)
    return ckks_set_error(CKKS_EUNSUPPORTED,
                          "%s: the fused kernel is not built or not schedulable for log_n=%d, level=%d "
                          "(built: log_n 10..13, level 2..7)", fn, ctx->log_n, level);
  CKKS_REQUIRE(out && ct_a && ct_b && key && scratch, "%s: NULL pointer argument", fn);
  const size_t need = ckks_ct_mul_scratch_bytes_3k(ctx, n_ct, level);
  CKKS_REQUIRE(scratch_bytes >= need, "%s: scratch of %zu bytes < %zu needed", fn, scratch_bytes,
               need);
  // default: one sub-batch per kPairsPerSub pairs, at most kMaxSub, from
  // 2 kPairsPerSub pairs on; sub-batch h runs on internal stream h mod 4
  const int split_req = ctx->tune_cm_split
                            ? ctx->tune_cm_split
                            : (n_ct >= 2 * kPairsPerSub ? (n_ct / kPairsPerSub < kMaxSub ? n_ct / kPairsPerSub : kMaxSub) : 1);
  int split = split_req < n_ct ? split_req : n_ct;
  if (max_split > 0 && split > max_split) split = max_split;
  cudaStream_t st = as_stream(stream);
  if (split <= 1) return cm_launch_one(ctx, out, ct_a, ct_b, key, n_ct, level, cm_carve(scratch, ctx->n, n_ct, level), st, fn);
  // Concurrent sub-batches: the kernels of one sub-batch fill the partial last
  // waves of another's and overlap the HBM-bound tensor product with the
  // compute-bound ModUp / ModDown.  Fork / join through events keeps the
  // caller's stream order (stream capture records them as graph edges).
  SplitStreams* ss = nullptr;
  if (int rc = split_streams_for_device(&ss, fn)) return rc;
  std::lock_guard<std::mutex> lock(ss->mu);
  cudaError_t e = cudaEventRecord(ss->fork, st);
  const size_t in_ct = (size_t)2 * level * ctx->n, out_ct = (size_t)2 * (level - 1) * ctx->n;
  unsigned char* sbase = reinterpret_cast<unsigned char*>(scratch);
  int rc = CKKS_OK;
  const int n_streams = split < kMaxSplit ? split : kMaxSplit;
  for (int h = 0; h < n_streams && e == cudaSuccess; ++h) e = cudaStreamWaitEvent(ss->s[h], ss->fork, 0);
  for (int h = 0; h < split && e == cudaSuccess && rc == CKKS_OK; ++h) {
    const int c0 = (int)((long long)n_ct * h / split), c1 = (int)((long long)n_ct * (h + 1) / split);
    const int m = c1 - c0;
    rc = cm_launch_one(ctx, out + (size_t)c0 * out_ct, ct_a + (size_t)c0 * in_ct, ct_b + (size_t)c0 * in_ct, key,
                       m, level, cm_carve(sbase, ctx->n, m, level), ss->s[h % n_streams], fn);
    sbase += cm_words(ctx->n, m, level) * sizeof(u64);
  }
  for (int h = 0; h < n_streams && e == cudaSuccess && rc == CKKS_OK; ++h) {
    e = cudaEventRecord(ss->join[h], ss->s[h]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ss->join[h], 0);
  }
  if (rc != CKKS_OK) return rc;
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  return CKKS_OK;
}

extern "C" int ckks_ct_mul_relin_rescale(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                                         const uint64_t* ct_b, const uint64_t* key, int n_ct,
                                         int level, void* scratch, size_t scratch_bytes,
                                         void* stream) {
  return ckks_ct_mul_launch(ctx, out, ct_a, ct_b, key, n_ct, level, scratch, scratch_bytes, stream,
                            "ckks_ct_mul_relin_rescale", 0, true);
}

extern "C" size_t ckks_rotate_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level) {
  return ckks_ct_mul_scratch_bytes_3k(ctx, n_ct, level);
}

extern "C" int ckks_rotate(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct, const uint64_t* key,
                           int n_ct, int level, uint64_t nu, void* scratch, size_t scratch_bytes,
                           void* stream) {
  const char* fn = "ckks_rotate";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(ctx->n_special == 1, "%s: context needs exactly one special prime", fn);
  CKKS_REQUIRE(level >= 1 && level <= ctx->n_q, "%s: level=%d outside [1, %d]", fn, level, ctx->n_q);
  CKKS_REQUIRE(ctx->log_n >= 6, "%s: log_n=%d below the supported minimum 6", fn, ctx->log_n);
  CKKS_REQUIRE(n_ct >= 0, "%s: n_ct < 0", fn);
  const u64 nu2n = nu & (2ull * ctx->n - 1);
  CKKS_REQUIRE(nu2n & 1, "%s: nu=%llu must be odd (a Galois element)", fn, (unsigned long long)nu);
  u64 pmin = ~0ull, pmax = 0;
  for (int i = 0; i < ctx->n_primes; ++i) {
    CKKS_REQUIRE(ctx->has_nega[i], "%s: prime %d has no 2N-th root", fn, i);
    pmin = ctx->primes[i] < pmin ? ctx->primes[i] : pmin;
    pmax = ctx->primes[i] > pmax ? ctx->primes[i] : pmax;
  }
  CKKS_REQUIRE(pmax < 2 * pmin, "%s: primes must satisfy max < 2 min (centred basis conversion)", fn);
  if (n_ct == 0) return CKKS_OK;
  CKKS_REQUIRE(out && ct && key && scratch, "%s: NULL pointer argument", fn);
  CKKS_REQUIRE(out != ct, "%s: out must differ from ct", fn);
  const size_t need = ckks_rotate_scratch_bytes(ctx, n_ct, level);
  CKKS_REQUIRE(scratch_bytes >= need, "%s: scratch of %zu bytes < %zu needed", fn, scratch_bytes, need);
  CmScratch S = cm_carve(scratch, ctx->n, n_ct, level);
  cudaStream_t st = as_stream(stream);
  return dispatch_cm(ctx->log_n, ctx->tune_cm_k, ctx->tune_cm_minb, [&]<int L, int K, int MINB>() -> int {
    using Sh = NttShape<L, K>;
    const int upc = ctx->tune_cm_upc ? ctx->tune_cm_upc : 1;
    const int smem_a = Sh::SMEM_WORDS * 8;
    const int smem_b = (Sh::SMEM_WORDS + 2 * Sh::N) * 8;
    const int smem_c = (Sh::SMEM_WORDS + Sh::N) * 8;
    if (int rc = require_smem(smem_b, L, fn)) return rc;
    auto ka = k_rot_prep<L, K, MINB>;
    auto kb = k_cm_modup<L, K, MINB>;
    auto kc = upc > 1 ? k_ks_down<L, K, MINB, true> : k_ks_down<L, K, MINB, false>;
    ensure_smem(ka, smem_a);
    ensure_smem(kb, smem_b);
    ensure_smem(kc, smem_c);
    {
      ProfSpan span(CKKS_STAGE_OTHER, st, "ckks rotation: automorphism + digits");
      const long long nu_a = (long long)n_ct * level;
      ka<<<grid1d((nu_a + upc - 1) / upc), Sh::T, smem_a, st>>>(reinterpret_cast<const u64*>(ct), S, level,
                                                                nu2n, ctx->d_pi, ctx->d_tw, n_ct, nu_a, upc);
    }
    if (int rc = ckks_check_launch(fn)) return rc;
    {
      ProfSpan span(CKKS_STAGE_CM_MODUP, st);
      const long long nu_b = (long long)n_ct * (level + 1);
      kb<<<grid1d((nu_b + upc - 1) / upc), Sh::T, smem_b, st>>>(
          S, reinterpret_cast<const double*>(key), level, ctx->n_q, ctx->d_pi, ctx->d_tw, n_ct, nu_b, upc);
    }
    if (int rc = ckks_check_launch(fn)) return rc;
    {
      ProfSpan span(CKKS_STAGE_CM_DOWN, st);
      const long long nu_c = (long long)n_ct * 2;
      kc<<<grid1d((nu_c + upc - 1) / upc), Sh::T, smem_c, st>>>(S, reinterpret_cast<u64*>(out), level, ctx->n_q,
                                                                ctx->d_pi, ctx->d_tw, ctx->d_pinv, nu_c, upc);
    }
    return ckks_check_launch(fn);
  }, fn);
}
