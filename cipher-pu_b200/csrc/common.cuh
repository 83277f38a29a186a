// common.cuh - shared types and exact 64-bit modular arithmetic for the
// CKKS evaluation core (sm_100a).
//
// Moduli are NTT-friendly primes below 2^47 (the production chain is 45-bit).
// The NTT butterflies run in exact FP64 (see ntt.cuh) with twiddles stored as
// (w, w / q) pairs; integer twiddle multiplications elsewhere use Shoup's
// precomputed quotient (w' = floor(w * 2^64 / q)), variable x variable
// products use Montgomery multiplication with R = 2^64 followed by a Shoup
// multiply by (R mod q).  All lazy integer ranges stay far inside 64 bits.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

typedef unsigned long long u64;
typedef long long i64;

struct TwPair {
  u64 w;   // twiddle
  u64 ws;  // floor(w * 2^64 / q)
};

// FP64 NTT twiddle: value and value / q (correctly rounded).
struct TwD {
  double w;
  double wq;
};

// Per-prime FP64 table slots ([n_primes][TWF_SLOTS][N] entries of TwD).
// Forward tables: psi^brv(m + i) for stage m = 2^s, group i < m, stored at
// m + i except in the stages of the transform's last register pass (the one
// with one butterfly block per thread), where group i = block * 2^u + grp is
// stored at m + grp * 2^S0 + block (S0 = first stage of that pass, u = s - S0)
// so that the 32 lanes of a warp read 32 consecutive entries.  The last pass
// depends on the register radix 2^K, so there is one forward table per K in
// {2, 3, 4, 5}; each is laid out for K' = min(K, log N), so K = 1 (log N = 1)
// reads the K = 2 table.
// Inverse tables: per stage s the h = N / 2^(s+1) twiddles omega^-(k 2^s),
// k < h, stored at h + k (one contiguous run per stage).
enum {
  TWF_FWD2 = 0,      // merged negacyclic forward, last-pass layout of K = 2
  TWF_FWD3 = 1,      // ... K = 3
  TWF_FWD4 = 2,      // ... K = 4
  TWF_FWD5 = 3,      // ... K = 5
  TWF_FWDC2 = 4,     // merged cyclic forward, K = 2 .. 5
  TWF_FWDC3 = 5,
  TWF_FWDC4 = 6,
  TWF_FWDC5 = 7,
  TWF_INV = 8,       // negacyclic inverse DIT twiddles (omega = psi^2), per stage
  TWF_INV_CYC = 9,   // cyclic inverse DIT twiddles, per stage
  TWF_POST = 10,     // N^-1 psi^-j, j in [0, N)
  TWF_POST_CYC = 11, // N^-1 (every j)
  TWF_SLOTS = 12
};

// Per-prime constants, one record per prime of a context.
struct PrimeInfo {
  u64 q, q2;
  u64 qlazy;      // 32 q: added before subtracting an NTT output (any value < 32 q)
  u64 mont_qinv;  // -q^{-1} mod 2^64
  u64 r_mod;      // 2^64 mod q
  u64 r_mod_s;    // Shoup companion of r_mod
  u64 one_s;      // floor(2^64 / q): Shoup companion of 1
  u64 ninv;       // N^{-1} mod q
  u64 ninv_s;
  u64 half;       // (q - 1) / 2 : centred representative boundary
  double qd;      // (double) q
  double qinv_d;  // 1.0 / q
};

// ------------------------------------------------------------------ modular
__device__ __forceinline__ u64 mulhi64(u64 a, u64 b) { return __umul64hi(a, b); }

// Shoup multiply, lazy: any y < 2^64, w < q, ws = floor(w 2^64 / q) -> [0, 2q)
__device__ __forceinline__ u64 shoup_lazy(u64 y, u64 w, u64 ws, u64 q) {
  const u64 qt = mulhi64(y, ws);
  return y * w - qt * q;
}

__device__ __forceinline__ u64 csub(u64 x, u64 m) { return x >= m ? x - m : x; }

__device__ __forceinline__ u64 shoup(u64 y, u64 w, u64 ws, u64 q) {
  return csub(shoup_lazy(y, w, ws, q), q);
}

// Montgomery product a*b*2^-64 mod q, lazy result in [0, 2q) when a*b < q*2^64.
__device__ __forceinline__ u64 mont_lazy(u64 a, u64 b, u64 q, u64 qinv_neg) {
  const u64 lo = a * b;
  const u64 hi = mulhi64(a, b);
  const u64 m = lo * qinv_neg;
  const u64 mqh = mulhi64(m, q);
  return hi + mqh + (lo != 0ull ? 1ull : 0ull);
}

// Exact a*b mod q for a, b < 2q (var x var) -> [0, q)
__device__ __forceinline__ u64 mulmod(u64 a, u64 b, const PrimeInfo& P) {
  const u64 t = mont_lazy(a, b, P.q, P.mont_qinv);      // a b R^-1, [0, 2q)
  return shoup(t, P.r_mod, P.r_mod_s, P.q);              // * R  -> a b
}

__device__ __forceinline__ u64 addmod(u64 a, u64 b, u64 q) { return csub(a + b, q); }
__device__ __forceinline__ u64 submod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + q - b; }

// Reduce any x < 2^64 to [0, q) (Shoup multiply by 1).
__device__ __forceinline__ u64 reduce_any(u64 x, const PrimeInfo& P) {
  return csub(shoup_lazy(x, 1ull, P.one_s, P.q), P.q);
}

// Reduce [0, 4q) -> [0, q)
__device__ __forceinline__ u64 reduce4(u64 x, u64 q, u64 q2) { return csub(csub(x, q2), q); }

__device__ __forceinline__ TwPair ldtw(const TwPair* p) {
  const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
  TwPair t;
  t.w = v.x;
  t.ws = v.y;
  return t;
}

__device__ __forceinline__ PrimeInfo ldpi(const PrimeInfo* p) { return *p; }

// ------------------------------------------------------------------ automorphism
// Evaluation slot i of the merged forward transform holds f(psi^(2 brv(i) + 1));
// psi_nu(f) = f(X^nu) at slot i is f at the slot returned here (nu odd, given
// mod 2N as nu2n).
__device__ __forceinline__ unsigned long long galois_eval_src(unsigned long long i, int log_n,
                                                              unsigned long long nu2n) {
  const unsigned long long n = 1ull << log_n;
  const unsigned long long b = __brev((unsigned)i) >> (32 - log_n);
  const unsigned long long e = ((2 * b + 1) * nu2n) & (2 * n - 1);
  return __brev((unsigned)((e - 1) >> 1)) >> (32 - log_n);
}

// ------------------------------------------------------------------ cache policy
// Polynomial limbs and key limbs are read once per CTA: load them without
// allocating in L1, so the L1 keeps the twiddle tables (loaded evict-last),
// which every transform of the CTA re-reads.
__device__ __forceinline__ u64 ld_stream(const u64* p) {
  u64 v;
  asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ ulonglong2 ld_stream2(const void* p) {
  ulonglong2 v;
  asm("ld.global.nc.L1::no_allocate.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_stream_d(const double* p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_stream2d(const void* p) {
  double2 v;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_keep2(const void* p) {
  double2 v;
  asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
