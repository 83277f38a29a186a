// ntt.cuh - one-CTA negacyclic / cyclic NTT over Z_q[X]/(X^N +- 1) for
// sm_100a, 64-bit coefficients, N = 2^LOGN.
//
// Each thread owns E = 2^K coefficients in registers.  The LOGN butterfly
// stages are grouped into passes of at most K stages; inside a pass all
// butterflies are register-local (radix-2^K), between passes the coefficients
// are exchanged through padded shared memory (one pad word per 16 / 32 words,
// which keeps the 64-bit accesses of every pass at the two-wavefront minimum).
//
// Forward: Cooley-Tukey, natural-order coefficients in, evaluations in
// bit-reversed order out; twiddle tw[m + i] for group i of stage m (merged
// psi form; Harvey lazy butterflies with values in [0, 4q)).
// Inverse: Gentleman-Sande with the inverse table, bit-reversed in, natural
// out, then * N^-1 (values in [0, 2q) throughout).
//
// Register layouts:
//   layout "C" (pass 0): thread t holds positions t + T*r        (coalesced)
//   layout "Z" (last pass): sub-problem g = t + T*c holds the contiguous run
//                          g * 2^kp + r                          (per-thread runs)
// The forward transform takes layout C and returns layout Z; the inverse
// takes Z and returns C.  Positions are element indices of the polynomial,
// so a caller may load / store in either layout without changing the data
// order in memory.
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
  __host__ __device__ static constexpr int last() { return NP; }
};

__device__ __forceinline__ int padix(int p, int sh) { return p + (p >> sh); }

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

// Position of register index e (0..E-1) in layout C / layout Z.
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

// ---------------------------------------------------------------- butterflies
// No per-butterfly reduction: with q < 2^47 the 64-bit words have room for
// the growth.  Forward (Cooley-Tukey): t = w y mod q lands in [0, 2q), so
// both outputs grow by at most 2q per stage (x + t, x + 2q - t); after the
// LOGN <= 14 stages a value below B_in is below B_in + 28q.  Inverse
// (Gentleman-Sande): the difference branch is re-reduced by the Shoup
// multiply to [0, 2q) while the sum branch at most doubles, so the input of
// the stage run d-th is below 2q * 2^d; the difference is offset by that
// bound (bs) to stay non-negative.  After LOGN stages values are below
// 2q * 2^14 < 2^62, and the closing N^-1 Shoup multiply accepts any word.
__device__ __forceinline__ void ct_bfly(u64& x, u64& y, const TwPair& w, u64 q, u64 q2) {
  const u64 t = shoup_lazy(y, w.w, w.ws, q);
  const u64 xr = x;
  x = xr + t;
  y = xr + q2 - t;
}

__device__ __forceinline__ void gs_bfly(u64& x, u64& y, const TwPair& w, u64 q, u64 bs) {
  const u64 u = x + y;
  const u64 v = x + bs - y;
  x = u;
  y = shoup_lazy(v, w.w, w.ws, q);
}

template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void fwd_pass(u64 (&x)[1 << K], int tid, const TwPair* __restrict__ tw,
                                         u64 q, u64 q2) {
  constexpr int N = 1 << LOGN;
  constexpr int T = N >> K;
  constexpr int BSZ = N >> S0;
  constexpr int DMIN = BSZ >> KP;
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
#pragma unroll
  for (int c = 0; c < SUBS; ++c) {
    const int g = tid + T * c;
    const int block = g / DMIN;
#pragma unroll
    for (int u = 0; u < KP; ++u) {
      const int half = RR >> (u + 1);
#pragma unroll
      for (int grp = 0; grp < (1 << u); ++grp) {
        const TwPair w = ldtw(tw + (1 << (S0 + u)) + block * (1 << u) + grp);
#pragma unroll
        for (int j = 0; j < half; ++j) {
          const int r = grp * 2 * half + j;
          ct_bfly(x[c * RR + r], x[c * RR + r + half], w, q, q2);
        }
      }
    }
  }
}

template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void inv_pass(u64 (&x)[1 << K], int tid, const TwPair* __restrict__ itw,
                                         u64 q, u64 q2) {
  constexpr int N = 1 << LOGN;
  constexpr int T = N >> K;
  constexpr int BSZ = N >> S0;
  constexpr int DMIN = BSZ >> KP;
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
#pragma unroll
  for (int c = 0; c < SUBS; ++c) {
    const int g = tid + T * c;
    const int block = g / DMIN;
#pragma unroll
    for (int u = KP - 1; u >= 0; --u) {
      const int half = RR >> (u + 1);
      const u64 bs = q2 << (LOGN - 1 - (S0 + u));  // input bound of this stage
#pragma unroll
      for (int grp = 0; grp < (1 << u); ++grp) {
        const TwPair w = ldtw(itw + (1 << (S0 + u)) + block * (1 << u) + grp);
#pragma unroll
        for (int j = 0; j < half; ++j) {
          const int r = grp * 2 * half + j;
          gs_bfly(x[c * RR + r], x[c * RR + r + half], w, q, bs);
        }
      }
    }
  }
}

template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void sm_store(const u64 (&x)[1 << K], u64* sm, int tid) {
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
  constexpr int SH = NttShape<LOGN, K>::PADSH;
#pragma unroll
  for (int c = 0; c < SUBS; ++c)
#pragma unroll
    for (int r = 0; r < RR; ++r) sm[padix(pass_pos<LOGN, K, S0, KP>(tid, c, r), SH)] = x[c * RR + r];
}

template <int LOGN, int K, int S0, int KP>
__device__ __forceinline__ void sm_load(u64 (&x)[1 << K], const u64* sm, int tid) {
  constexpr int SUBS = 1 << (K - KP);
  constexpr int RR = 1 << KP;
  constexpr int SH = NttShape<LOGN, K>::PADSH;
#pragma unroll
  for (int c = 0; c < SUBS; ++c)
#pragma unroll
    for (int r = 0; r < RR; ++r) x[c * RR + r] = sm[padix(pass_pos<LOGN, K, S0, KP>(tid, c, r), SH)];
}

// forward passes 1..NP (pass 0 done by caller-side helper below)
template <int LOGN, int K, int P>
struct FwdRest {
  __device__ __forceinline__ static void run(u64 (&x)[1 << K], u64* sm, int tid,
                                             const TwPair* __restrict__ tw, u64 q, u64 q2) {
    using S = NttShape<LOGN, K>;
    if constexpr (P <= S::NP) {
      sm_store<LOGN, K, S::s0(P - 1), S::kp(P - 1)>(x, sm, tid);
      __syncthreads();
      sm_load<LOGN, K, S::s0(P), S::kp(P)>(x, sm, tid);
      __syncthreads();
      fwd_pass<LOGN, K, S::s0(P), S::kp(P)>(x, tid, tw, q, q2);
      FwdRest<LOGN, K, P + 1>::run(x, sm, tid, tw, q, q2);
    }
  }
};

// inverse passes NP..1 (descending), then pass 0
template <int LOGN, int K, int P>
struct InvRest {
  __device__ __forceinline__ static void run(u64 (&x)[1 << K], u64* sm, int tid,
                                             const TwPair* __restrict__ itw, u64 q, u64 q2) {
    using S = NttShape<LOGN, K>;
    if constexpr (P >= 1) {
      inv_pass<LOGN, K, S::s0(P), S::kp(P)>(x, tid, itw, q, q2);
      sm_store<LOGN, K, S::s0(P), S::kp(P)>(x, sm, tid);
      __syncthreads();
      sm_load<LOGN, K, S::s0(P - 1), S::kp(P - 1)>(x, sm, tid);
      __syncthreads();
      InvRest<LOGN, K, P - 1>::run(x, sm, tid, itw, q, q2);
    }
  }
};

// Forward NTT: x in layout C with values below 4q -> layout Z, values below
// 4q + 2q LOGN <= 32q (see the butterfly notes); callers that subtract a
// transformed value add LAZY_FWD_BOUND(q) first.
__device__ __forceinline__ u64 lazy_fwd_bound(u64 q) { return q << 5; }

template <int LOGN, int K>
__device__ __forceinline__ void ntt_fwd_lazy(u64 (&x)[1 << K], u64* sm, int tid,
                                             const TwPair* __restrict__ tw, u64 q, u64 q2) {
  fwd_pass<LOGN, K, 0, K>(x, tid, tw, q, q2);
  FwdRest<LOGN, K, 1>::run(x, sm, tid, tw, q, q2);
}

// Forward NTT with the result reduced to [0, q).
template <int LOGN, int K>
__device__ __forceinline__ void ntt_fwd(u64 (&x)[1 << K], u64* sm, int tid,
                                        const TwPair* __restrict__ tw, const PrimeInfo& P) {
  ntt_fwd_lazy<LOGN, K>(x, sm, tid, tw, P.q, P.q2);
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) x[e] = reduce_any(x[e], P);
}

// Inverse NTT: x in layout Z with values in [0, 2q) -> layout C, values in [0, q),
// multiplied by N^-1.
template <int LOGN, int K>
__device__ __forceinline__ void ntt_inv(u64 (&x)[1 << K], u64* sm, int tid,
                                        const TwPair* __restrict__ itw, const PrimeInfo& P) {
  InvRest<LOGN, K, NttShape<LOGN, K>::NP>::run(x, sm, tid, itw, P.q, P.q2);
  inv_pass<LOGN, K, 0, K>(x, tid, itw, P.q, P.q2);
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) x[e] = csub(shoup_lazy(x[e], P.ninv, P.ninv_s, P.q), P.q);
}

// Layout-Z global access: the last pass has unit stride inside each run, so
// registers (e, e+1) with e even are adjacent words; move them as 16-byte vectors.
template <int LOGN, int K>
__device__ __forceinline__ void load_z(u64 (&x)[1 << K], const u64* __restrict__ src, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); e += 2) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(src + posZ<LOGN, K>(tid, e)));
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
  for (int e = 0; e < (1 << K); ++e) x[e] = __ldg(src + posC<LOGN, K>(tid, e));
}
template <int LOGN, int K>
__device__ __forceinline__ void store_c(const u64 (&x)[1 << K], u64* __restrict__ dst, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) dst[posC<LOGN, K>(tid, e)] = x[e];
}

// Layout-Z global access: the last pass has unit stride inside each run, so
// registers (e, e+1) with e even are adjacent words; move them as 16-byte vectors.
template <int LOGN, int K>
__device__ __forceinline__ void load_z(u64 (&x)[1 << K], const u64* __restrict__ src, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); e += 2) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(src + posZ<LOGN, K>(tid, e)));
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
  for (int e = 0; e < (1 << K); ++e) x[e] = __ldg(src + posC<LOGN, K>(tid, e));
}
template <int LOGN, int K>
__device__ __forceinline__ void store_c(const u64 (&x)[1 << K], u64* __restrict__ dst, int tid) {
#pragma unroll
  for (int e = 0; e < (1 << K); ++e) dst[posC<LOGN, K>(tid, e)] = x[e];
}

// Dynamic shared memory bytes needed by one transform.
template <int LOGN, int K>
constexpr int ntt_smem_bytes() {
  return NttShape<LOGN, K>::SMEM_WORDS * 8;
}
