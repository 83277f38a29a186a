// encode.cu - CKKS slot encoding / decoding (FP64 canonical embedding),
// encryption, decryption and the DARE decrypt-reencrypt refresh.
//
// Slot convention (as the reference's negacyclic DFT): slot k < N/2 is the
// evaluation of the message polynomial at Phi^(2k+1), Phi = exp(i pi / N);
// its conjugate sits at index N-1-k.
//   encode: V (Hermitian completed) -> m_j = Re(Phi^-j FFT(V)[j]) / N,
//           coefficient = round(Delta m_j), reduced per limb.
//   decode: coefficients (balanced CRT over the limbs) -> x_j / Delta ->
//           V[k] = sum_j x_j Phi^j e^{+2 pi i jk / N}.
// The FFT is an in-shared-memory radix-2 transform, one CTA per polynomial.
#include "dispatch.cuh"
#include "profile.hpp"

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {__fma_rn(a.re, b.re, -a.im * b.im), __fma_rn(a.re, b.im, a.im * b.re)};
}

// In-place FFT of N = 2^LOGN points in shared memory, natural order in and out.
// sign = -1: X[k] = sum x_j e^{-2 pi i jk/N};  sign = +1: e^{+...}.
template <int LOGN>
__device__ void smem_fft(cplx* a, int sign) {
  constexpr int N = 1 << LOGN;
  const int tid = threadIdx.x, nt = blockDim.x;
  // bit-reversal permutation
  for (int i = tid; i < N; i += nt) {
    const int j = (int)(__brev((unsigned)i) >> (32 - LOGN));
    if (i < j) {
      const cplx t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
  __syncthreads();
  for (int s = 1; s <= LOGN; ++s) {
    const int m = 1 << s, half = m >> 1;
    for (int b = tid; b < N / 2; b += nt) {
      const int grp = b / half, k = b % half;
      const int i0 = grp * m + k, i1 = i0 + half;
      double sn, cs;
      sincospi((double)(2 * k) / (double)m, &sn, &cs);
      const cplx w = {cs, sign * sn};
      const cplx t = cmul(w, a[i1]);
      const cplx u = a[i0];
      a[i0] = {u.re + t.re, u.im + t.im};
      a[i1] = {u.re - t.re, u.im - t.im};
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- encode
template <int LOGN>
__global__ void k_encode(u64* __restrict__ out, const double* __restrict__ slots, int n_slots,
                         int level, double scale, const PrimeInfo* __restrict__ pi) {
  extern __shared__ cplx fa[];
  constexpr int N = 1 << LOGN;
  const long long poly = blockIdx.x;
  const int tid = threadIdx.x, nt = blockDim.x;
  const double* sp = slots + (size_t)poly * n_slots * 2;
  for (int k = tid; k < N; k += nt) fa[k] = {0.0, 0.0};
  __syncthreads();
  for (int k = tid; k < n_slots; k += nt) {
    const cplx v = {scale * sp[2 * k], scale * sp[2 * k + 1]};
    fa[k] = v;
    const int c = N - 1 - k;
    if (c != k && c >= n_slots) fa[c] = {v.re, -v.im};
  }
  __syncthreads();
  smem_fft<LOGN>(fa, -1);
  u64* o = out + (size_t)poly * level * N;
  for (int j = tid; j < N; j += nt) {
    double sn, cs;
    sincospi(-(double)j / (double)N, &sn, &cs);
    const double mj = (fa[j].re * cs - fa[j].im * sn) / (double)N;  // Re(Phi^-j X_j) / N
    const double r = rint(mj);
    const long long iv = (long long)r;
    for (int i = 0; i < level; ++i) {
      const u64 q = pi[i].q;
      long long t = iv % (long long)q;
      if (t < 0) t += (long long)q;
      o[(size_t)i * N + j] = (u64)t;
    }
  }
}

// ---------------------------------------------------------------- decode
// Balanced mixed-radix (Garner) reconstruction of the centred integer from its
// residues, evaluated in double: x = sum_k v_k P_k, |v_k| <= (q_k - 1) / 2.
struct CrtConsts {
  int level;
  u64 q[16];
  TwPair pinv[16];      // (q_0 ... q_{k-1})^-1 mod q_k
  TwPair pmod[16][16];  // P_m mod q_k  (P_m = q_0 ... q_{m-1}), m < k
  double pd[16];        // P_k as double
};

__device__ __forceinline__ double crt_to_double(const u64* r, const CrtConsts& C) {
  long long v[16];
  double x = 0.0;
  for (int k = 0; k < C.level; ++k) {
    const u64 q = C.q[k];
    // t = (r_k - sum_{m<k} v_m P_m) * P_k^-1 mod q
    u64 acc = r[k] % q;
    for (int m = 0; m < k; ++m) {
      const u64 vm = v[m] >= 0 ? (u64)v[m] : (u64)(v[m] + (long long)q);
      acc = submod(acc, shoup(vm, C.pmod[k][m].w, C.pmod[k][m].ws, q), q);
    }
    const u64 t = k ? shoup(acc, C.pinv[k].w, C.pinv[k].ws, q) : acc;
    v[k] = t > (q - 1) / 2 ? (long long)t - (long long)q : (long long)t;
    x = fma((double)v[k], C.pd[k], x);
  }
  return x;
}

template <int LOGN>
__global__ void k_decode(double* __restrict__ slots, const u64* __restrict__ in, int n_slots,
                         double inv_scale, CrtConsts C) {
  extern __shared__ cplx fa[];
  constexpr int N = 1 << LOGN;
  const long long poly = blockIdx.x;
  const int tid = threadIdx.x, nt = blockDim.x;
  const u64* src = in + (size_t)poly * C.level * N;
  for (int j = tid; j < N; j += nt) {
    u64 r[16];
    for (int k = 0; k < C.level; ++k) r[k] = src[(size_t)k * N + j];
    const double x = crt_to_double(r, C) * inv_scale;
    double sn, cs;
    sincospi((double)j / (double)N, &sn, &cs);
    fa[j] = {x * cs, x * sn};  // x_j Phi^j
  }
  __syncthreads();
  smem_fft<LOGN>(fa, +1);
  double* o = slots + (size_t)poly * n_slots * 2;
  for (int k = tid; k < n_slots; k += nt) {
    o[2 * k] = fa[k].re;
    o[2 * k + 1] = fa[k].im;
  }
}

static int make_crt(const ckks_ctx* ctx, int level, CrtConsts& C, const char* fn) {
  CKKS_REQUIRE(level >= 1 && level <= 16 && level <= ctx->n_primes, "%s: level=%d unsupported", fn,
               level);
  C.level = level;
  double pd = 1.0;
  for (int k = 0; k < level; ++k) {
    const u64 q = ctx->primes[k];
    C.q[k] = q;
    C.pd[k] = pd;
    u64 pk = 1;  // P_k mod q
    for (int m = 0; m < k; ++m) {
      u64 pm = 1;  // P_m mod q
      for (int t = 0; t < m; ++t) pm = h_mulmod(pm, ctx->primes[t] % q, q);
      C.pmod[k][m] = h_twp(pm, q);
      pk = h_mulmod(pk, ctx->primes[m] % q, q);
    }
    C.pinv[k] = h_twp(k ? h_invmod(pk, q) : 1, q);
    pd *= (double)q;
  }
  return CKKS_OK;
}

template <int LOGN>
static int fft_threads() {
  return (1 << LOGN) >= 1024 ? 512 : ((1 << LOGN) / 2 > 32 ? (1 << LOGN) / 2 : 32);
}

// dispatch over log_n in [2, 13] for the FFT kernels
template <typename F>
static int dispatch_fft(int log_n, F&& f, const char* fn) {
  switch (log_n) {
#define CKKS_FFT_CASE(L) \
  case L:                \
    return f.template operator()<L>();
    CKKS_FFT_CASE(2)
    CKKS_FFT_CASE(3)
    CKKS_FFT_CASE(4)
    CKKS_FFT_CASE(5)
    CKKS_FFT_CASE(6)
    CKKS_FFT_CASE(7)
    CKKS_FFT_CASE(8)
    CKKS_FFT_CASE(9)
    CKKS_FFT_CASE(10)
    CKKS_FFT_CASE(11)
    CKKS_FFT_CASE(12)
    CKKS_FFT_CASE(13)
#undef CKKS_FFT_CASE
    default:
      return ckks_set_error(CKKS_EUNSUPPORTED, "%s: log_n=%d outside [2, 13]", fn, log_n);
  }
}

extern "C" int ckks_encode(const ckks_ctx* ctx, uint64_t* out, const double* slots, int n_polys,
                           int n_slots, int level, double scale, void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks encode");
  const char* fn = "ckks_encode";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_slots >= 0 && n_slots <= ctx->n / 2, "%s: n_slots=%d outside [0, N/2]", fn, n_slots);
  CKKS_REQUIRE(level >= 1 && level <= ctx->n_primes, "%s: level=%d outside [1, %d]", fn, level,
               ctx->n_primes);
  CKKS_REQUIRE(scale > 0.0 && scale < 9.0e15, "%s: scale must lie in (0, 2^53)", fn);
  for (int i = 0; i < level; ++i)
    CKKS_REQUIRE(ctx->has_nega[i], "%s: prime %d has no 2N-th root", fn, i);
  if (n_polys <= 0) return CKKS_OK;
  cudaStream_t st = as_stream(stream);
  int rc = dispatch_fft(ctx->log_n, [&]<int L>() -> int {
    const int smem = (1 << L) * (int)sizeof(cplx);
    ensure_smem(k_encode<L>, smem);
    k_encode<L><<<grid1d(n_polys), fft_threads<L>(), smem, st>>>(
        reinterpret_cast<u64*>(out), slots, n_slots, level, scale, ctx->d_pi);
    return ckks_check_launch(fn);
  }, fn);
  if (rc) return rc;
  return ckks_ntt(ctx, out, n_polys, 0, level, 0, 0, stream);
}

extern "C" int ckks_decode(const ckks_ctx* ctx, double* slots, const uint64_t* in_coef, int n_polys,
                           int n_slots, int level, double scale, void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks decode");
  const char* fn = "ckks_decode";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_slots >= 0 && n_slots <= ctx->n / 2, "%s: n_slots=%d outside [0, N/2]", fn, n_slots);
  CKKS_REQUIRE(scale > 0.0, "%s: scale must be positive", fn);
  CrtConsts C;
  if (int rc = make_crt(ctx, level, C, fn)) return rc;
  if (n_polys <= 0) return CKKS_OK;
  cudaStream_t st = as_stream(stream);
  return dispatch_fft(ctx->log_n, [&]<int L>() -> int {
    const int smem = (1 << L) * (int)sizeof(cplx);
    ensure_smem(k_decode<L>, smem);
    k_decode<L><<<grid1d(n_polys), fft_threads<L>(), smem, st>>>(
        slots, reinterpret_cast<const u64*>(in_coef), n_slots, 1.0 / scale, C);
    return ckks_check_launch(fn);
  }, fn);
}

// ---------------------------------------------------------------- decrypt
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_decrypt(u64* __restrict__ out, const u64* __restrict__ ct, const u64* __restrict__ s_eval,
              int level, const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  const long long c = blockIdx.x / level;
  const int i = blockIdx.x % level;
  const int tid = threadIdx.x;
  const PrimeInfo P = pi[i];
  const size_t LN = (size_t)level * N;
  const u64* c0 = ct + c * 2 * LN + (size_t)i * N;
  u64 x[Sh::E], y[Sh::E], s[Sh::E];
  load_c<LOGN, K>(x, c0, tid);
  load_c<LOGN, K>(y, c0 + LN, tid);
  load_c<LOGN, K>(s, s_eval + (size_t)i * N, tid);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) x[e] = addmod(x[e], mulmod(y[e], s[e], P), P.q);
  c_to_z<LOGN, K>(x, sm, tid);
  ntt_inv<LOGN, K>(x, sm, tid, twbase<LOGN>(tw, i), P);
  store_c<LOGN, K>(x, out + c * LN + (size_t)i * N, tid);
}

extern "C" int ckks_decrypt(const ckks_ctx* ctx, uint64_t* out_coef, const uint64_t* ct,
                            const uint64_t* s_eval, int n_ct, int level, void* stream) {
  const char* fn = "ckks_decrypt";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(level >= 1 && level <= ctx->n_primes, "%s: level=%d outside [1, %d]", fn, level,
               ctx->n_primes);
  for (int i = 0; i < level; ++i)
    CKKS_REQUIRE(ctx->has_nega[i], "%s: prime %d has no 2N-th root", fn, i);
  if (n_ct <= 0) return CKKS_OK;
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    if constexpr (K < 1) {
      return ckks_set_error(CKKS_EUNSUPPORTED, "%s: N too small", fn);
    } else {
      using Sh = NttShape<L, K>;
      ensure_smem(k_decrypt<L, K>, Sh::SMEM_WORDS * 8);
      k_decrypt<L, K><<<grid1d((long long)n_ct * level), Sh::T, Sh::SMEM_WORDS * 8, as_stream(stream)>>>(
          reinterpret_cast<u64*>(out_coef), reinterpret_cast<const u64*>(ct),
          reinterpret_cast<const u64*>(s_eval), level, ctx->d_pi, ctx->d_tw);
      return ckks_check_launch(fn);
    }
  });
}

// ---------------------------------------------------------------- encrypt
template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_encrypt(u64* __restrict__ out, const u64* __restrict__ m_eval, const u64* __restrict__ s_eval,
              const u64* __restrict__ a, const long long* __restrict__ err, int level,
              const PrimeInfo* __restrict__ pi, const TwD* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  const long long c = blockIdx.x / level;
  const int i = blockIdx.x % level;
  const int tid = threadIdx.x;
  const PrimeInfo P = pi[i];
  const size_t LN = (size_t)level * N;
  u64 x[Sh::E];
  const long long* ep = err + c * N;
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) {
    long long v = ep[posC<LOGN, K>(tid, e)] % (long long)P.q;
    x[e] = (u64)(v < 0 ? v + (long long)P.q : v);
  }
  ntt_fwd<LOGN, K>(x, sm, tid, twbase<LOGN>(tw, i), P);
  z_to_c<LOGN, K>(x, sm, tid);
  u64 av[Sh::E], sv[Sh::E];
  load_c<LOGN, K>(av, a + c * LN + (size_t)i * N, tid);
  load_c<LOGN, K>(sv, s_eval + (size_t)i * N, tid);
  if (m_eval) {
    u64 mv[Sh::E];
    load_c<LOGN, K>(mv, m_eval + c * LN + (size_t)i * N, tid);
#pragma unroll
    for (int e = 0; e < Sh::E; ++e) x[e] = addmod(x[e], mv[e], P.q);
  }
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) x[e] = submod(x[e], mulmod(av[e], sv[e], P), P.q);
  u64* o0 = out + c * 2 * LN + (size_t)i * N;
  store_c<LOGN, K>(x, o0, tid);
  store_c<LOGN, K>(av, o0 + LN, tid);
}

extern "C" int ckks_encrypt(const ckks_ctx* ctx, uint64_t* out, const uint64_t* m_eval,
                            const uint64_t* s_eval, const uint64_t* a, const int64_t* e, int n_ct,
                            int level, void* stream) {
  const char* fn = "ckks_encrypt";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(level >= 1 && level <= ctx->n_primes, "%s: level=%d outside [1, %d]", fn, level,
               ctx->n_primes);
  for (int i = 0; i < level; ++i)
    CKKS_REQUIRE(ctx->has_nega[i], "%s: prime %d has no 2N-th root", fn, i);
  if (n_ct <= 0) return CKKS_OK;
  CKKS_REQUIRE(out && s_eval && a && e, "%s: NULL pointer argument", fn);
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    using Sh = NttShape<L, K>;
    ensure_smem(k_encrypt<L, K>, Sh::SMEM_WORDS * 8);
    k_encrypt<L, K><<<grid1d((long long)n_ct * level), Sh::T, Sh::SMEM_WORDS * 8, as_stream(stream)>>>(
        reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(m_eval),
        reinterpret_cast<const u64*>(s_eval), reinterpret_cast<const u64*>(a),
        reinterpret_cast<const long long*>(e), level, ctx->d_pi, ctx->d_tw);
    return ckks_check_launch(fn);
  });
}

// ---------------------------------------------------------------- DARE
// Step 1: dec_i = INTT(c0_i + c1_i s_i) into scratch (coefficient domain) -- k_decrypt.
// Step 2: per (ct, output limb j): balanced CRT of dec over the input limbs,
//         optional rounding shift m = round(x / 2^shift), then
//         out0_j = NTT_j([m + e]_{q_j}) - a_j s_j,  out1_j = a_j.
struct DareConsts {
  CrtConsts crt;
  u64 p128_lo[16], p128_hi[16];  // P_k mod 2^128
  u64 pkq[16][16];               // P_k mod q_j (output limb j)
  int shift;
};

__device__ __forceinline__ void crt_digits(const u64* r, const CrtConsts& C, long long* v) {
  for (int k = 0; k < C.level; ++k) {
    const u64 q = C.q[k];
    u64 acc = r[k] % q;
    for (int m = 0; m < k; ++m) {
      const u64 vm = v[m] >= 0 ? (u64)v[m] : (u64)(v[m] + (long long)q);
      acc = submod(acc, shoup(vm, C.pmod[k][m].w, C.pmod[k][m].ws, q), q);
    }
    const u64 t = k ? shoup(acc, C.pinv[k].w, C.pinv[k].ws, q) : acc;
    v[k] = t > (q - 1) / 2 ? (long long)t - (long long)q : (long long)t;
  }
}

template <int LOGN, int K>
__global__ void __launch_bounds__(NttShape<LOGN, K>::T)
    k_dare_out(u64* __restrict__ out, const u64* __restrict__ dec, const u64* __restrict__ s_eval,
               const u64* __restrict__ a, const long long* __restrict__ err, int level_in,
               int level_out, DareConsts D, const PrimeInfo* __restrict__ pi,
               const TwD* __restrict__ tw) {
  extern __shared__ u64 sm[];
  using Sh = NttShape<LOGN, K>;
  constexpr int N = Sh::N;
  const long long c = blockIdx.x / level_out;
  const int j = blockIdx.x % level_out;
  const int tid = threadIdx.x;
  const PrimeInfo P = pi[j];
  const u64* dsrc = dec + c * (size_t)level_in * N;
  u64 x[Sh::E];
#pragma unroll 1
  for (int e = 0; e < Sh::E; ++e) {
    const int pos = posC<LOGN, K>(tid, e);
    u64 r[16];
    long long v[16];
    for (int k = 0; k < level_in; ++k) r[k] = dsrc[(size_t)k * N + pos];
    crt_digits(r, D.crt, v);
    const long long ev = err[c * N + pos];
    const u64 evq = ev >= 0 ? reduce_any((u64)ev, P) : submod(0, reduce_any((u64)(-ev), P), P.q);
    u64 res;
    if (D.shift == 0) {
      // x mod q_j = sum_k v_k (P_k mod q_j), exact for any |x| < Q / 2
      u64 s = evq;
      for (int k = 0; k < level_in; ++k) {
        const u64 mag = reduce_any((u64)(v[k] >= 0 ? v[k] : -v[k]), P);
        const u64 vk = v[k] >= 0 ? mag : submod(0, mag, P.q);
        s = addmod(s, mulmod(vk, D.pkq[k][j], P), P.q);
      }
      res = s;
    } else {
      // x as a signed 128-bit integer (exact when |x| < 2^127), then a rounded
      // arithmetic shift, then reduction mod q_j through (hi, lo) words.
      unsigned __int128 xs = 0;
      for (int k = 0; k < level_in; ++k) {
        const unsigned __int128 pk128 = ((unsigned __int128)D.p128_hi[k] << 64) | D.p128_lo[k];
        xs += (unsigned __int128)(__int128)v[k] * pk128;
      }
      __int128 xv = (__int128)xs;
      xv = (xv + ((__int128)1 << (D.shift - 1))) >> D.shift;  // round half up
      const bool neg = xv < 0;
      const unsigned __int128 mag = neg ? (unsigned __int128)(-xv) : (unsigned __int128)xv;
      const u64 hi = (u64)(mag >> 64), lo = (u64)mag;
      u64 r = addmod(mulmod(reduce_any(hi, P), P.r_mod, P), reduce_any(lo, P), P.q);
      if (neg) r = submod(0, r, P.q);
      res = addmod(r, evq, P.q);
    }
    x[e] = res;
  }
  ntt_fwd<LOGN, K>(x, sm, tid, twbase<LOGN>(tw, j), P);
  z_to_c<LOGN, K>(x, sm, tid);
  const size_t LN = (size_t)level_out * N;
  u64 av[Sh::E], sv[Sh::E];
  load_c<LOGN, K>(av, a + c * LN + (size_t)j * N, tid);
  load_c<LOGN, K>(sv, s_eval + (size_t)j * N, tid);
#pragma unroll
  for (int e = 0; e < Sh::E; ++e) x[e] = submod(x[e], mulmod(av[e], sv[e], P), P.q);
  u64* o0 = out + c * 2 * LN + (size_t)j * N;
  store_c<LOGN, K>(x, o0, tid);
  store_c<LOGN, K>(av, o0 + LN, tid);
}

extern "C" size_t ckks_dare_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level_in) {
  if (!ctx || n_ct < 0 || level_in < 1) return 0;
  return (size_t)n_ct * level_in * ctx->n * sizeof(u64);
}

extern "C" int ckks_dare_refresh(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct,
                                 const uint64_t* s_eval, const uint64_t* a_fresh,
                                 const int64_t* e_fresh, int n_ct, int level_in, int level_out,
                                 int shift_bits, void* scratch, size_t scratch_bytes, void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks DARE refresh");
  const char* fn = "ckks_dare_refresh";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(level_in >= 1 && level_in <= 16 && level_in <= ctx->n_primes,
               "%s: level_in=%d unsupported", fn, level_in);
  CKKS_REQUIRE(level_out >= 1 && level_out <= ctx->n_primes, "%s: level_out=%d unsupported", fn,
               level_out);
  CKKS_REQUIRE(shift_bits >= 0 && shift_bits < 100, "%s: shift_bits=%d outside [0, 100)", fn,
               shift_bits);
  CKKS_REQUIRE(out != ct, "%s: out must differ from ct", fn);
  if (n_ct <= 0) return CKKS_OK;
  CKKS_REQUIRE(scratch_bytes >= ckks_dare_scratch_bytes(ctx, n_ct, level_in),
               "%s: scratch too small (%zu < %zu)", fn, scratch_bytes,
               ckks_dare_scratch_bytes(ctx, n_ct, level_in));
  DareConsts D;
  if (int rc = make_crt(ctx, level_in, D.crt, fn)) return rc;
  CKKS_REQUIRE(level_out <= 16, "%s: level_out=%d above 16", fn, level_out);
  unsigned __int128 pk = 1;
  for (int k = 0; k < level_in; ++k) {
    D.p128_lo[k] = (u64)pk;
    D.p128_hi[k] = (u64)(pk >> 64);
    pk *= ctx->primes[k];  // mod 2^128
    for (int j = 0; j < level_out; ++j) {
      const u64 qj = ctx->primes[j];
      u64 v = 1;
      for (int m = 0; m < k; ++m) v = h_mulmod(v, ctx->primes[m] % qj, qj);
      D.pkq[k][j] = v;
    }
  }
  D.shift = shift_bits;
  if (int rc = ckks_decrypt(ctx, reinterpret_cast<uint64_t*>(scratch), ct, s_eval, n_ct, level_in,
                            stream))
    return rc;
  return dispatch_logn(ctx->log_n, [&]<int L, int K>() -> int {
    using Sh = NttShape<L, K>;
    ensure_smem(k_dare_out<L, K>, Sh::SMEM_WORDS * 8);
    k_dare_out<L, K><<<grid1d((long long)n_ct * level_out), Sh::T, Sh::SMEM_WORDS * 8,
                       as_stream(stream)>>>(
        reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(scratch),
        reinterpret_cast<const u64*>(s_eval), reinterpret_cast<const u64*>(a_fresh),
        reinterpret_cast<const long long*>(e_fresh), level_in, level_out, D, ctx->d_pi, ctx->d_tw);
    return ckks_check_launch(fn);
  });
}
