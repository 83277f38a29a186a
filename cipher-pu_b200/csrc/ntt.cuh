// ntt.cuh - one-CTA negacyclic / cyclic NTT over Z_q[X]/(X^N +- 1) for
// sm_100a, N = 2^LOGN, primes q < 2^47.
//
// Arithmetic: exact FP64.  Residues below 2^52 are exact doubles; a twiddle
// product y * w mod q is formed as hi = y w (rounded) plus lo = fma(y, w, -hi)
// (the exact rounding error), the quotient qt = round(y * (w / q)) comes from
// one FMA against 1.5 * 2^52, and r = fma(-qt, q, hi) + lo is exact with
// |r| <= q.  On B200 this double-word product runs at twice the rate of the
// integer Shoup product (measured by ckks_modmul_peak), and the butterflies
// need no integer compare / select at all: values are kept signed and lazy.
//
// Each thread owns E = 2^K coefficients in registers.  The LOGN butterfly
// stages are grouped into passes of at most K stages; inside a pass all
// butterflies are register-local (radix-2^K), between passes the coefficients
// are exchanged through padded shared memory (one pad word per 16 / 32 words,
// which keeps the 64-bit accesses of every pass at the two-wavefront minimum).
//
// Forward: Cooley-Tukey, natural-order coefficients in, evaluations in
// bit-reversed order out; twiddle tw[m + i] for group i of stage m (merged
// psi form).  |x| grows by at most q per stage.
// Inverse: the input is the bit-reversed evaluation vector, so the cyclic
// inverse DFT is a decimation-in-time Cooley-Tukey (distance 1, 2, ... N/2,
// pair (p, p + h) with twiddle omega^-(p mod h) * N/(2h)); the negacyclic
// untwist psi^-j and N^-1 are one closing multiply by post[j] = N^-1 psi^-j.
// Growth is again at most q per stage, so nothing is reduced until the end.
//
// Register layouts:
//   layout "C" (pass 0): thread t holds positions t + T*r        (coalesced)
//   layout "Z" (last pass): sub-problem g = t + T*c holds the contiguous run
//                          g * 2^kp + r                          (per-thread runs)
// The forward transform takes layout C and returns layout Z; the inverse
// takes Z and returns C.  Positions are element indices of the polynomial,
// so a caller may load / store in either layout without changing the data
// order in memory.  Both transforms take canonical residues in [0, q) (the
// forward also accepts any value below 4q) and return canonical residues.
#pragma once
#include "common.cuh"

template <int LOGN, int K>
struct NttShape {
  static constexpr int N = 1 << LOGN;
  static constexpr int E = 1 << K;
  static constexpr int T = N >> K;
  static constexpr int R = LOGN - K;                      // stages after pass 0
  static constexpr int NP = (R + K - 1) / K;               // further passes
  static constexpr int PADSH = (K >= 5) ? 5 : 4;
  static constexpr int SMEM_WORDS = N + (N >> PADSH);
  __host__ __device__ static constexpr int kp(int p) {
    return p == 0 ? K : (R / NP + ((p - 1) < (R % NP) ? 1 : 0));
  }
  __host__ __device__ static constexpr int s0(int p) {
    int s = 0;
    for (int i = 0; i < p; ++i) s += kp(i);
    return s;
  }
};

__device__ __forceinline__ int padix(int p, int sh) { return p + (p >> sh); }

// Barrier of the T threads that run one transform.  Every kernel but one
// launches exactly T threads per CTA, where this is a CTA-wide barrier; the
// persistent batch kernel runs two N = 2^12 transforms (T = 256) side by side
// in a 512-thread CTA, each group on its own named barrier 1 + threadIdx.x / T.
// Below one warp (T < 32, tiny rings) the hardware needs the CTA barrier.
template <int T>
__device__ __forceinline__ void group_sync() {
  if constexpr (T < 32) {
    __syncthreads();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / T)), "n"(T) : "memory");
  }
}

// position of register (c, r) of a pass that starts at stage S0 with KP stages
template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ int pass_pos(int tid, int c, int r) {
  constexpr int N = 1 << LOGN;
  constexpr int T = N >> K;
  constexpr int BSZ = N >> S0;
  constexpr int DMIN = BSZ >> KP;
  const int g = tid + T * c;
  const int block = g / DMIN;
  const int off = g % DMIN;
  return block * BSZ + off + DMIN * r;
}

template <int LOGN, int K>
__device__ __forceinline__ int posC(int tid, int e) {
  return tid + (NttShape<LOGN, K>::T) * e;
}
template <int LOGN, int K>
__device__ __forceinline__ int posZ(int tid, int e) {
  using S = NttShape<LOGN, K>;
  constexpr int P = S::NP;
  constexpr int KP = S::kp(P);
  constexpr int S0 = S::s0(P);
  return pass_pos<LOGN, K, S0, KP>(tid, e >> KP, e & ((1 << KP) - 1));
}

// ---------------------------------------------------------------- FP64 modular arithmetic
#define CKKS_FP_MAGIC 6755399441055744.0  // 1.5 * 2^52: fma(a, b, M) - M = round(a b)
#define CKKS_FP_TWO52 4503599627370496.0

__device__ __forceinline__ TwD ldtwd(const TwD* p) {
  const double2 v = ld_keep2(p);
  TwD t;
  t.w = v.x;
  t.wq = v.y;
  return t;
}

// y * w mod q up to a multiple of q: exact, |result| <= q, for |y| < 2^51.
__device__ __forceinline__ double fmulmod(double y, double w, double wq, double qd) {
  const double hi = __dmul_rn(y, w);
  const double lo = __fma_rn(y, w, -hi);
  const double qt = __dadd_rn(__fma_rn(y, wq, CKKS_FP_MAGIC), -CKKS_FP_MAGIC);
  return __dadd_rn(__fma_rn(-qt, qd, hi), lo);
}

// a * b mod q up to a multiple of q for exact integers |a|, |b| < 4q
// (q < 2^47): hi + lo is the exact product, qt = round(hi / q) is off by at
// most 1/16 (|a b| / q < 2^49, two roundings of 2^-53), so hi - qt q is an
// exact integer below 0.57 q in magnitude and |result| < 0.57 q + ulp(hi) / 2
// < 2^48.
__device__ __forceinline__ double fmulmod_var(double a, double b, double qd, double qinv) {
  const double hi = __dmul_rn(a, b);
  const double lo = __fma_rn(a, b, -hi);
  const double qt = __dadd_rn(__fma_rn(hi, qinv, CKKS_FP_MAGIC), -CKKS_FP_MAGIC);
  return __dadd_rn(__fma_rn(-qt, qd, hi), lo);
}

// u64 residue (< 2^52) -> exact double
__device__ __forceinline__ double u2d(u64 x) {
  return __dadd_rn(__longlong_as_double((long long)(x | 0x4330000000000000ull)), -CKKS_FP_TWO52);
}

// exact integer double with |x| < 2^51 -> the congruent integer of
// magnitude <= q / 2 + 1 (still a double)
__device__ __forceinline__ double dreduce(double x, double qd, double qinv) {
  const double qt = __dadd_rn(__fma_rn(x, qinv, CKKS_FP_MAGIC), -CKKS_FP_MAGIC);
  return __fma_rn(-qt, qd, x);
}

// exact integer double with |x| < 2^51 -> canonical residue in [0, q)
__device__ __forceinline__ u64 d2canon(double x, double qd, double qinv) {
  const double qt = __dadd_rn(__fma_rn(x, qinv, CKKS_FP_MAGIC), -CKKS_FP_MAGIC);
  double r = __fma_rn(-qt, qd, x);  // |r| <= q/2 + 1
  r = r < 0.0 ? __dadd_rn(r, qd) : r;
  r = r >= qd ? __dadd_rn(r, -qd) : r;
  return (u64)__double_as_longlong(__dadd_rn(r, CKKS_FP_TWO52)) & 0x000FFFFFFFFFFFFFull;
}

// ---------------------------------------------------------------- passes
__device__ __forceinline__ void ct_bfly_fp(double& x, double& y, const TwD& w, double qd) {
  const double t = fmulmod(y, w.w, w.wq, qd);
  const double xr = x;
  x = __dadd_rn(xr, t);
  y = __dadd_rn(xr, -t);
}

// forward pass: stages S0 .. S0+KP-1, group-uniform twiddles (group
// i = block * 2^u + grp of stage m = 2^(S0+u)); in the last pass the table
// holds that group at m + grp * 2^S0 + block (lane-contiguous, see common.cuh)
template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void fwd_pass(double (&x)[1 << K], int tid, const TwD* __restrict__ tw,
                                         double qd) {
  constexpr int N = 1 << LOGN;
  constexpr int T = N >> K;
  constexpr int BSZ = N >> S0;
  constexpr int DMIN = BSZ >> KP;
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
  constexpr bool LAST = S0 + KP == LOGN;
#pragma unroll
  for (int c = 0; c < SUBS; ++c) {
    const int g = tid + T * c;
    const int block = g / DMIN;
#pragma unroll
    for (int u = 0; u < KP; ++u) {
      const int half = RR >> (u + 1);
#pragma unroll
      for (int grp = 0; grp < (1 << u); ++grp) {
        const int ti = LAST ? (1 << (S0 + u)) + grp * (1 << S0) + block
                            : (1 << (S0 + u)) + block * (1 << u) + grp;
        const TwD w = ldtwd(tw + ti);
#pragma unroll
        for (int j = 0; j < half; ++j) {
          const int r = grp * 2 * half + j;
          ct_bfly_fp(x[c * RR + r], x[c * RR + r + half], w, qd);
        }
      }
    }
  }
}

// inverse (DIT) pass: stages S0+KP-1 down to S0 (distances ascending);
// the pair (p, p + h) at stage s, h = N >> (s + 1), uses omega^-((p mod h) 2^s),
// stored at itw[h + (p mod h)]
template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void inv_pass(double (&x)[1 << K], int tid, const TwD* __restrict__ itw,
                                         double qd) {
  constexpr int N = 1 << LOGN;
  constexpr int T = N >> K;
  constexpr int BSZ = N >> S0;
  constexpr int DMIN = BSZ >> KP;
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
#pragma unroll
  for (int c = 0; c < SUBS; ++c) {
    const int g = tid + T * c;
    const int off = g % DMIN;
#pragma unroll
    for (int u = KP - 1; u >= 0; --u) {
      const int half = RR >> (u + 1);
      const int s = S0 + u;
#pragma unroll
      for (int j = 0; j < half; ++j) {
        const TwD w = ldtwd(itw + (N >> (s + 1)) + off + DMIN * j);
#pragma unroll
        for (int grp = 0; grp < (1 << u); ++grp) {
          const int r = grp * 2 * half + j;
          ct_bfly_fp(x[c * RR + r], x[c * RR + r + half], w, qd);
        }
      }
    }
  }
}

template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void sm_store(const double (&x)[1 << K], double* sm, int tid) {
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
  constexpr int SH = NttShape<LOGN, K>::PADSH;
#pragma unroll
  for (int c = 0; c < SUBS; ++c)
#pragma unroll
    for (int r = 0; r < RR; ++r) sm[padix(pass_pos<LOGN, K, S0, KP>(tid, c, r), SH)] = x[c * RR + r];
}

template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void sm_load(double (&x)[1 << K], const double* sm, int tid) {
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
  constexpr int SH = NttShape<LOGN, K>::PADSH;
#pragma unroll
  for (int c = 0; c < SUBS; ++c)
#pragma unroll
    for (int r = 0; r < RR; ++r) x[c * RR + r] = sm[padix(pass_pos<LOGN, K, S0, KP>(tid, c, r), SH)];
}

template <int LOGN, int K, int P>
struct FwdRest {
  __device__ __forceinline__ static void run(double (&x)[1 << K], double* sm, int tid,
                                             const TwD* __restrict__ tw, double qd) {
    using S = NttShape<LOGN, K>;
    if constexpr (P <= S::NP) {
      sm_store<LOGN, K, S::s0(P - 1), S::kp(P - 1)>(x, sm, tid);
      group_sync<S::T>();
      sm_load<LOGN, K, S::s0(P), S::kp(P)>(x, sm, tid);
      group_sync<S::T>();
      fwd_pass<LOGN, K, S::s0(P), S::kp(P)>(x, tid, tw, qd);
      FwdRest<LOGN, K, P + 1>::run(x, sm, tid, tw, qd);
    }
  }
};

template <int LOGN, int K, int P>
struct InvRest {
  __device__ __forceinline__ static void run(double (&x)[1 << K], double* sm, int tid,
                                             const TwD* __restrict__ itw, double qd) {
    using S = NttShape<LOGN, K>;
    if constexpr (P >= 1) {
      inv_pass<LOGN, K, S::s0(P), S::kp(P)>(x, tid, itw, qd);
      sm_store<LOGN, K, S::s0(P), S::kp(P)>(x, sm, tid);
      group_sync<S::T>();
      sm_load<LOGN, K, S::s0(P - 1), S::kp(P - 1)>(x, sm, tid);
      group_sync<S::T>();
      InvRest<LOGN, K, P - 1>::run(x, sm, tid, itw, qd);
    }
  }
};

// Per-prime table base: tb = tw + prime * TWF_SLOTS * N.
template <int LOGN>
__device__ __forceinline__ const TwD* twbase(const TwD* tw, int prime) {
  return tw + (size_t)prime * TWF_SLOTS * (1 << LOGN);
}

// Forward NTT on exact doubles: layout C in (integers of magnitude < 4q),
// layout Z out, unreduced: |result| < 4q + 0.75 q LOGN < 2^51 (an input to
// fmulmod or d2canon as it stands).
template <int LOGN, int K>
__device__ __forceinline__ void ntt_fwd_d(double (&d)[1 << K], u64* sm, int tid,
                                          const TwD* __restrict__ tb, const PrimeInfo& P,
                                          bool cyclic = false) {
  constexpr int N = 1 << LOGN;
  static_assert(K >= 1 && K <= 5, "forward twiddle layouts exist for K <= 5");
  constexpr int kslot = K <= 2 ? 0 : K - 2;  // K = 1 only at log N = 1, where the K = 2 layout is the same
  const TwD* tw = tb + ((cyclic ? TWF_FWDC2 : TWF_FWD2) + kslot) * N;
  double* smd = reinterpret_cast<double*>(sm);
  fwd_pass<LOGN, K, 0, K>(d, tid, tw, P.qd);
  FwdRest<LOGN, K, 1>::run(d, smd, tid, tw, P.qd);
}

// Forward NTT: layout C in (values < 4q), layout Z out, canonical [0, q).
template <int LOGN, int K>
__device__ __forceinline__ void ntt_fwd(u64 (&x)[1 << K], u64* sm, int tid, const TwD* __restrict__ tb,
                                        const PrimeInfo& P, bool cyclic = false) {
  double d[1 << K];
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) d[e] = u2d(x[e]);
  ntt_fwd_d<LOGN, K>(d, sm, tid, tb, P, cyclic);
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) x[e] = d2canon(d[e], P.qd, P.qinv_d);
}

// Inverse NTT (with N^-1) on exact doubles: layout Z in (|d| <= 1.5 q),
// layout C out in x, canonical.  Each stage adds at most q to the magnitude,
// so |d| stays below (1.5 + log N) q < 2^51 for q < 2^47.
template <int LOGN, int K>
__device__ __forceinline__ void ntt_inv_d(double (&d)[1 << K], u64 (&x)[1 << K], u64* sm, int tid,
                                          const TwD* __restrict__ tb, const PrimeInfo& P, bool cyclic = false) {
  constexpr int N = 1 << LOGN;
  const TwD* itw = tb + (cyclic ? TWF_INV_CYC : TWF_INV) * N;
  const TwD* post = tb + (cyclic ? TWF_POST_CYC : TWF_POST) * N;
  double* smd = reinterpret_cast<double*>(sm);
  InvRest<LOGN, K, NttShape<LOGN, K>::NP>::run(d, smd, tid, itw, P.qd);
  inv_pass<LOGN, K, 0, K>(d, tid, itw, P.qd);
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) {
    const TwD pw = ldtwd(post + posC<LOGN, K>(tid, e));
    x[e] = d2canon(fmulmod(d[e], pw.w, pw.wq, P.qd), P.qd, P.qinv_d);
  }
}

// Inverse NTT (with N^-1): layout Z in (canonical), layout C out, canonical.
template <int LOGN, int K>
__device__ __forceinline__ void ntt_inv(u64 (&x)[1 << K], u64* sm, int tid, const TwD* __restrict__ tb,
                                        const PrimeInfo& P, bool cyclic = false) {
  double d[1 << K];
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) d[e] = u2d(x[e]);
  ntt_inv_d<LOGN, K>(d, x, sm, tid, tb, P, cyclic);
}

// Layout-Z global access: the last pass has unit stride inside each run, so
// registers (e, e+1) with e even are adjacent words; move them as 16-byte vectors.
template <int LOGN, int K>
__device__ __forceinline__ void load_z(u64 (&x)[1 << K], const u64* __restrict__ src, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); e += 2) {
    const ulonglong2 v = ld_stream2(src + posZ<LOGN, K>(tid, e));
    x[e] = v.x;
    x[e + 1] = v.y;
  }
}
template <int LOGN, int K>
__device__ __forceinline__ void store_z(const u64 (&x)[1 << K], u64* __restrict__ dst, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); e += 2)
    *reinterpret_cast<ulonglong2*>(dst + posZ<LOGN, K>(tid, e)) = make_ulonglong2(x[e], x[e + 1]);
}
template <int LOGN, int K>
__device__ __forceinline__ void load_c(u64 (&x)[1 << K], const u64* __restrict__ src, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) x[e] = ld_stream(src + posC<LOGN, K>(tid, e));
}
template <int LOGN, int K>
__device__ __forceinline__ void store_c(const u64 (&x)[1 << K], u64* __restrict__ dst, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) dst[posC<LOGN, K>(tid, e)] = x[e];
}

// Register re-distribution through the transform's shared buffer: layout Z
// (the forward output) to layout C (lane-contiguous, for coalesced global
// access and elementwise work against naturally ordered operands), and back
// (the inverse input).  Callers must not have threads still reading sm (every
// transform returns with sm free); both end with a barrier.
template <int LOGN, int K, typename V>
__device__ __forceinline__ void z_to_c(V (&x)[1 << K], u64* sm, int tid) {
  using S = NttShape<LOGN, K>;
  V* sv = reinterpret_cast<V*>(sm);
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) sv[padix(posZ<LOGN, K>(tid, e), S::PADSH)] = x[e];
  group_sync<S::T>();
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) x[e] = sv[padix(posC<LOGN, K>(tid, e), S::PADSH)];
  group_sync<S::T>();
}
template <int LOGN, int K, typename V>
__device__ __forceinline__ void c_to_z(V (&x)[1 << K], u64* sm, int tid) {
  using S = NttShape<LOGN, K>;
  V* sv = reinterpret_cast<V*>(sm);
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) sv[padix(posC<LOGN, K>(tid, e), S::PADSH)] = x[e];
  group_sync<S::T>();
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) x[e] = sv[padix(posZ<LOGN, K>(tid, e), S::PADSH)];
  group_sync<S::T>();
}

// Dynamic shared memory bytes needed by one transform.
template <int LOGN, int K>
constexpr int ntt_smem_bytes() {
  return NttShape<LOGN, K>::SMEM_WORDS * 8;
}
