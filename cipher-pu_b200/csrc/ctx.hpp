// ctx.hpp - host-side context of the CKKS evaluation core: the prime basis of
// one ring dimension with its device-resident twiddle tables and constants.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/ckks_b200.h"
#include "common.cuh"

struct ckks_ctx {
  int log_n = 0;
  int n = 0;
  int n_primes = 0;
  int n_special = 0;  // trailing special primes (0 or 1)
  int n_q = 0;        // n_primes - n_special
  int device = 0;
  int tune_cm_k = 0;     // ct-mult: log2 coefficients per thread (0 = default)
  int tune_cm_minb = 0;  // ct-mult: register budget, 1 balanced / 2 tight (0 = default)
  int tune_cm_split = 0; // ct-mult: concurrent sub-batches, 1..4 (0 = default)
  int tune_ntt_k = 0;    // ckks_ntt: log2 coefficients per thread, 2..5 (0 = default)
  int tune_cm_upc = 0;   // ct-mult / rotation: work units per CTA, 1..8 (0 = default 1)
  int tune_cm_tma = 0;   // ct-mult tensor kernel: 1 = persistent TMA-fed, 2 = one CTA per unit (0 = default)
  int tune_wait_cycles = 0;  // limit of every bounded device wait, SM cycles (0 = default, ~1 s)
  int tune_cm_fused = 0;     // ct-mult: 0 = fused kernel where built, 1 = fused required, 2 = three kernels
  int tune_cm_tmem = 0;      // ct-mult ModUp accumulators: 0 = default, 1 = TMEM where built, 2 = shared memory
  std::vector<u64> primes, psi, omega;
  std::vector<int> has_nega;
  std::vector<PrimeInfo> h_pi;
  PrimeInfo* d_pi = nullptr;  // [n_primes]
  TwD* d_tw = nullptr;        // [n_primes][TWF_SLOTS][n]: FP64 NTT tables (common.cuh)
  TwPair* d_pinv = nullptr;   // [n_q]: special^-1 mod q_i (zeros when n_special == 0)
  TwPair* d_qtinv = nullptr;  // [n_q][n_q]: q_t^-1 mod q_i at [t][i], i < t
  TwPair* d_misc = nullptr;   // [n_primes][4]: (1, one_s) helpers; slot 1: R mod q
  unsigned char* d_ntt_tc = nullptr;  // tensor-core transform tables (ntt_tc.cu), built on first use
  double scale = 0.0, sigma = 0.0;  // scheme constants of ckks_ctx_create_params (not read by kernels)
  u64 seed = 0;
  std::vector<std::vector<u64>> h_qtinv;  // host copies
  std::vector<u64> h_pinv;
};

// ---------------------------------------------------------------- errors
int ckks_set_error(int code, const char* fmt, ...);
int ckks_check_launch(const char* what);

#define CKKS_REQUIRE(cond, ...)                                  \
  do {                                                           \
    if (!(cond)) return ckks_set_error(CKKS_EINVAL, __VA_ARGS__); \
  } while (0)

// ---------------------------------------------------------------- host math
static inline u64 h_mulmod(u64 a, u64 b, u64 q) {
  return (u64)(((unsigned __int128)a * b) % q);
}
static inline u64 h_powmod(u64 b, u64 e, u64 q) {
  u64 r = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) r = h_mulmod(r, b, q);
    b = h_mulmod(b, b, q);
    e >>= 1;
  }
  return r;
}
static inline u64 h_invmod(u64 a, u64 q) { return h_powmod(a % q, q - 2, q); }  // q prime
static inline u64 h_shoup(u64 w, u64 q) { return (u64)(((unsigned __int128)w << 64) / q); }
static inline TwD h_twd(u64 w, u64 q) {
  TwD t;
  t.w = (double)(w % q);
  t.wq = t.w / (double)q;
  return t;
}
static inline TwPair h_twp(u64 w, u64 q) {
  TwPair t;
  t.w = w % q;
  t.ws = h_shoup(t.w, q);
  return t;
}

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Limit, in SM cycles, of the bounded device-side waits of this context's
// kernels (2^31 - 1 cycles by default: about 1.1 s at the 1965 MHz boost clock).
static inline long long ckks_wait_limit(const ckks_ctx* ctx) {
  return ctx->tune_wait_cycles > 0 ? (long long)ctx->tune_wait_cycles : 2147483647ll;
}
