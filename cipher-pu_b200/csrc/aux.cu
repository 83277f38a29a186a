// aux.cu - noise monitor reductions, slot SNR, block sparsity, RNS split /
// merge and the energy-threshold gear controller.
#include "dispatch.cuh"
#include "profile.hpp"

// ---------------------------------------------------------------- noise energy
// Per row: exact 128-bit sum of min(c, q - c)^2 (rtl/m4/noise_monitor.sv:42-78).
__global__ void k_noise_energy(unsigned long long* __restrict__ out, const u64* __restrict__ in,
                               int row_len, u64 q) {
  const long long row = blockIdx.x;
  const u64* src = in + (size_t)row * row_len;
  unsigned __int128 acc = 0;
  for (int i = threadIdx.x; i < row_len; i += blockDim.x) {
    const u64 c = src[i] % q;
    const u64 a = c <= q - c ? c : q - c;
    acc += (unsigned __int128)a * a;
  }
  u64 lo = (u64)acc, hi = (u64)(acc >> 64);
  // warp reduction on (hi, lo) with carry
  for (int off = 16; off; off >>= 1) {
    const u64 olo = __shfl_down_sync(0xffffffffu, lo, off);
    const u64 ohi = __shfl_down_sync(0xffffffffu, hi, off);
    const u64 nlo = lo + olo;
    hi += ohi + (nlo < lo ? 1 : 0);
    lo = nlo;
  }
  __shared__ u64 slo[32], shi[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    slo[w] = lo;
    shi[w] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    u64 tlo = 0, thi = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      const u64 nlo = tlo + slo[k];
      thi += shi[k] + (nlo < tlo ? 1 : 0);
      tlo = nlo;
    }
    out[2 * row] = tlo;
    out[2 * row + 1] = thi;
  }
}

extern "C" int ckks_noise_energy(uint64_t* out_sum, const uint64_t* in, int n_rows, int row_len,
                                 uint64_t q, void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks noise monitor");
  CKKS_REQUIRE(n_rows >= 0 && row_len >= 0, "ckks_noise_energy: negative size");
  CKKS_REQUIRE(q >= 2 && q < (1ull << 62), "ckks_noise_energy: q outside [2, 2^62)");
  if (n_rows == 0) return CKKS_OK;
  k_noise_energy<<<grid1d(n_rows), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<unsigned long long*>(out_sum), reinterpret_cast<const u64*>(in), row_len, q);
  return ckks_check_launch("ckks_noise_energy");
}

// ---------------------------------------------------------------- noise energy, saturating
// The same sum with the RTL accumulator's saturation flag
// (rtl/m4/noise_monitor.sv:62-73: an ACC_W-bit accumulator that stops, flag
// set, once a sum would wrap).  The sum is formed exactly in 192 bits
// (q < 2^62: each square < 2^122, at most 2^31 terms), so the flag does not
// depend on the order of the parallel reduction: saturated[row] = 1 exactly
// when the sum reaches 2^acc_bits, and the reported sum is then clamped to
// 2^acc_bits - 1 (the RTL holds its last pre-wrap value instead, which
// depends on the coefficient order).
struct U192 {
  u64 w0, w1, w2;
};
__device__ __forceinline__ void add192(U192& a, const U192& b) {
  const u64 s0 = a.w0 + b.w0;
  const u64 c0 = s0 < a.w0 ? 1ull : 0ull;
  const u64 t1 = a.w1 + b.w1;
  const u64 c1a = t1 < a.w1 ? 1ull : 0ull;
  const u64 s1 = t1 + c0;
  const u64 c1b = s1 < t1 ? 1ull : 0ull;
  a.w0 = s0;
  a.w1 = s1;
  a.w2 = a.w2 + b.w2 + c1a + c1b;
}

__global__ void k_noise_energy_sat(unsigned long long* __restrict__ out, unsigned char* __restrict__ sat,
                                   const u64* __restrict__ in, int row_len, u64 q, int acc_bits) {
  const long long row = blockIdx.x;
  const u64* src = in + (size_t)row * row_len;
  U192 acc = {0, 0, 0};
  for (int i = threadIdx.x; i < row_len; i += blockDim.x) {
    const u64 c = src[i] % q;
    const u64 a = c <= q - c ? c : q - c;
    const U192 sq = {a * a, __umul64hi(a, a), 0};
    add192(acc, sq);
  }
  for (int off = 16; off; off >>= 1) {
    const U192 o = {__shfl_down_sync(0xffffffffu, acc.w0, off), __shfl_down_sync(0xffffffffu, acc.w1, off),
                    __shfl_down_sync(0xffffffffu, acc.w2, off)};
    add192(acc, o);
  }
  __shared__ U192 part[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) part[w] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    U192 tot = {0, 0, 0};
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) add192(tot, part[k]);
    // tot >= 2^acc_bits ?
    bool over;
    if (acc_bits >= 128) over = tot.w2 != 0;
    else if (acc_bits >= 64) over = tot.w2 != 0 || (acc_bits < 128 && (tot.w1 >> (acc_bits - 64)) != 0);
    else over = tot.w2 != 0 || tot.w1 != 0 || (tot.w0 >> acc_bits) != 0;
    if (over) {
      tot.w0 = acc_bits >= 64 ? ~0ull : ((1ull << acc_bits) - 1);
      tot.w1 = acc_bits >= 128 ? ~0ull : (acc_bits > 64 ? ((1ull << (acc_bits - 64)) - 1) : 0ull);
    }
    out[2 * row] = tot.w0;
    out[2 * row + 1] = tot.w1;
    sat[row] = over ? 1 : 0;
  }
}

extern "C" int ckks_noise_energy_sat(uint64_t* out_sum, uint8_t* saturated, const uint64_t* in, int n_rows,
                                     int row_len, uint64_t q, int acc_bits, void* stream) {
  CKKS_REQUIRE(n_rows >= 0 && row_len >= 0, "ckks_noise_energy_sat: negative size");
  CKKS_REQUIRE(q >= 2 && q < (1ull << 62), "ckks_noise_energy_sat: q outside [2, 2^62)");
  CKKS_REQUIRE(acc_bits >= 1 && acc_bits <= 128, "ckks_noise_energy_sat: acc_bits=%d outside [1, 128]",
               acc_bits);
  if (n_rows == 0) return CKKS_OK;
  CKKS_REQUIRE(out_sum && saturated && in, "ckks_noise_energy_sat: NULL pointer argument");
  k_noise_energy_sat<<<grid1d(n_rows), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<unsigned long long*>(out_sum), reinterpret_cast<unsigned char*>(saturated),
      reinterpret_cast<const u64*>(in), row_len, q, acc_bits);
  return ckks_check_launch("ckks_noise_energy_sat");
}

// ---------------------------------------------------------------- slot SNR
// Per row: sum |ref|^2 and sum |dec - ref|^2 over row_len complex values.
__global__ void k_snr(double* __restrict__ out, const double* __restrict__ dec,
                      const double* __restrict__ ref, int row_len, int complex_vals) {
  const long long row = blockIdx.x;
  const int stride = complex_vals ? 2 : 1;
  const double* d = dec + (size_t)row * row_len * stride;
  const double* r = ref + (size_t)row * row_len * stride;
  double s = 0.0, e = 0.0;
  for (int i = threadIdx.x; i < row_len * stride; i += blockDim.x) {
    const double rv = r[i], dv = d[i];
    s = fma(rv, rv, s);
    e = fma(dv - rv, dv - rv, e);
  }
  for (int off = 16; off; off >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, off);
    e += __shfl_down_sync(0xffffffffu, e, off);
  }
  __shared__ double ss[32], se[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    ss[w] = s;
    se[w] = e;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ts = 0.0, te = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      ts += ss[k];
      te += se[k];
    }
    out[2 * row] = ts;
    out[2 * row + 1] = te;
  }
}

extern "C" int ckks_snr_sums(double* out, const double* dec, const double* ref, int n_rows,
                             int row_len, int complex_vals, void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks SNR probe sums");
  CKKS_REQUIRE(n_rows >= 0 && row_len >= 0, "ckks_snr_sums: negative size");
  if (n_rows == 0) return CKKS_OK;
  k_snr<<<grid1d(n_rows), 256, 0, as_stream(stream)>>>(out, dec, ref, row_len, complex_vals);
  return ckks_check_launch("ckks_snr_sums");
}

// ---------------------------------------------------------------- block sparsity
// Flat blocks of B weights whose max |w| < threshold are zeroed
// (scripts/exp_e10_sparsity_sweep_v2.py:102); keep[b] = 1 for kept blocks.
__global__ void k_block_mask_f64(double* __restrict__ out, unsigned char* __restrict__ keep,
                                 const double* __restrict__ w, long long n_blocks, int B,
                                 double threshold) {
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n_blocks) return;
  double m = 0.0;
  for (int i = 0; i < B; ++i) m = fmax(m, fabs(w[b * B + i]));
  const bool k = !(m < threshold);
  if (keep) keep[b] = k ? 1 : 0;
  for (int i = 0; i < B; ++i) out[b * B + i] = k ? w[b * B + i] : 0.0;
}

extern "C" int ckks_block_sparse_mask(double* out, uint8_t* keep, const double* w, int64_t n,
                                      int block, double threshold, void* stream) {
  CKKS_REQUIRE(n >= 0 && block >= 1, "ckks_block_sparse_mask: bad size");
  const long long nb = n / block;
  if (nb == 0) return CKKS_OK;
  k_block_mask_f64<<<grid1d((nb + 255) / 256), 256, 0, as_stream(stream)>>>(out, keep, w, nb, block,
                                                                           threshold);
  if (int rc = ckks_check_launch("ckks_block_sparse_mask")) return rc;
  const long long tail = n - nb * block;  // trailing partial block is kept as is
  if (tail > 0 && out != w) {
    cudaError_t e = cudaMemcpyAsync(out + nb * block, w + nb * block, tail * sizeof(double),
                                    cudaMemcpyDeviceToDevice, as_stream(stream));
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_block_sparse_mask: %s", cudaGetErrorString(e));
  }
  return CKKS_OK;
}

// Coefficient-domain block skip of the approximate multiplier
// (scripts/verify_m4_d_approx_mult.py:50 post_process_block): blocks of B
// residues whose max min(x, q - x) < threshold are zeroed; per-row skip counts.
__global__ void k_block_post(u64* __restrict__ out, int* __restrict__ skipped,
                             const u64* __restrict__ in, int row_len, int B, u64 q, u64 threshold,
                             int use_approx) {
  const long long row = blockIdx.x;
  const u64* src = in + (size_t)row * row_len;
  u64* dst = out + (size_t)row * row_len;
  const int nb = (row_len + B - 1) / B;
  int cnt = 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int lo = b * B, hi = min(row_len, lo + B);
    u64 m = 0;
    for (int i = lo; i < hi; ++i) {
      const u64 x = src[i];
      const u64 a = x < q - x ? x : q - x;
      m = a > m ? a : m;
    }
    const bool kill = use_approx && threshold != 0 && m < threshold;
    cnt += kill ? 1 : 0;
    for (int i = lo; i < hi; ++i) dst[i] = kill ? 0 : src[i];
  }
  for (int off = 16; off; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
  __shared__ int sc[32];
  if ((threadIdx.x & 31) == 0) sc[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0 && skipped) {
    int t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sc[k];
    skipped[row] = t;
  }
}

extern "C" int ckks_block_post_process(uint64_t* out, int32_t* skipped, const uint64_t* in,
                                       int n_rows, int row_len, int block, uint64_t q,
                                       uint64_t threshold, int use_approx, void* stream) {
  CKKS_REQUIRE(n_rows >= 0 && row_len >= 0, "ckks_block_post_process: negative size");
  CKKS_REQUIRE(q >= 2, "ckks_block_post_process: q < 2");
  if (n_rows == 0) return CKKS_OK;
  const int B = block <= 0 ? 1 : (block > row_len ? row_len : block);
  k_block_post<<<grid1d(n_rows), 128, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), skipped, reinterpret_cast<const u64*>(in), row_len, B > 0 ? B : 1,
      q, threshold, use_approx);
  return ckks_check_launch("ckks_block_post_process");
}

// ---------------------------------------------------------------- RNS split / merge
struct RnsConsts {
  int k, words;
  u64 p[8];
  TwPair r64[8];       // 2^64 mod p_i (Shoup), for word-wise reduction
  TwPair pinv[8];      // (p_0 ... p_{i-1})^-1 mod p_i
  TwPair pmod[8][8];   // (p_0 ... p_{m-1}) mod p_i, m < i
  u64 pw[8][8];        // P_m = p_0 ... p_{m-1} as `words` little-endian words
  u64 mw[8];           // M = p_0 ... p_{k-1}
  u64 hw[8];           // (M - 1) / 2
};

__device__ __forceinline__ u64 red_words(const u64* x, int words, u64 p, const TwPair& r64) {
  // Horner from the top word: acc = acc * 2^64 + w  (mod p)
  u64 acc = 0;
  for (int i = words - 1; i >= 0; --i) {
    const u64 t = csub(shoup_lazy(acc, r64.w, r64.ws, p), p);  // acc * 2^64 mod p
    acc = addmod(t, x[i] % p, p);
  }
  return acc;
}

__global__ void k_rns_split(u64* __restrict__ out, const u64* __restrict__ in, long long n,
                            RnsConsts C, int centered) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  u64 w[8];
  for (int i = 0; i < C.words; ++i) w[i] = in[idx * C.words + i];
  const bool neg = centered && (w[C.words - 1] >> 63);
  if (neg) {  // two's complement magnitude
    u64 carry = 1;
    for (int i = 0; i < C.words; ++i) {
      const u64 v = ~w[i] + carry;
      carry = (carry && v == 0) ? 1 : 0;
      w[i] = v;
    }
  }
  for (int k = 0; k < C.k; ++k) {
    const u64 r = red_words(w, C.words, C.p[k], C.r64[k]);
    out[(size_t)k * n + idx] = neg ? submod(0, r, C.p[k]) : r;
  }
}

__global__ void k_rns_merge(u64* __restrict__ out, const u64* __restrict__ in, long long n,
                            RnsConsts C, int centered) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  u64 v[8];
  for (int k = 0; k < C.k; ++k) {
    const u64 p = C.p[k];
    u64 acc = in[(size_t)k * n + idx] % p;
    for (int m = 0; m < k; ++m) acc = submod(acc, shoup(v[m] % p, C.pmod[k][m].w, C.pmod[k][m].ws, p), p);
    v[k] = k ? shoup(acc, C.pinv[k].w, C.pinv[k].ws, p) : acc;
  }
  // x = sum v_k P_k as a multiword integer in [0, M)
  u64 x[8];
  for (int i = 0; i < C.words; ++i) x[i] = 0;
  for (int k = 0; k < C.k; ++k) {
    u64 carry = 0;
    for (int i = 0; i < C.words; ++i) {
      const u64 lo = C.pw[k][i] * v[k];
      const u64 hi = __umul64hi(C.pw[k][i], v[k]);
      u64 s = x[i] + lo;
      u64 c1 = s < lo ? 1 : 0;
      s += carry;
      c1 += (s < carry) ? 1 : 0;
      x[i] = s;
      carry = hi + c1;
    }
  }
  if (centered) {  // x > (M - 1) / 2  ->  x - M (two's complement)
    bool gt = false;
    for (int i = C.words - 1; i >= 0; --i) {
      if (x[i] != C.hw[i]) {
        gt = x[i] > C.hw[i];
        break;
      }
    }
    if (gt) {
      u64 borrow = 0;
      for (int i = 0; i < C.words; ++i) {
        const u64 d = x[i] - C.mw[i] - borrow;
        borrow = (x[i] < C.mw[i] || (x[i] == C.mw[i] && borrow)) ? 1 : 0;
        x[i] = d;
      }
    }
  }
  for (int i = 0; i < C.words; ++i) out[idx * C.words + i] = x[i];
}

static void mw_mul_small(u64* x, int words, u64 m) {
  unsigned __int128 carry = 0;
  for (int i = 0; i < words; ++i) {
    const unsigned __int128 t = (unsigned __int128)x[i] * m + carry;
    x[i] = (u64)t;
    carry = t >> 64;
  }
}

static int make_rns(const uint64_t* primes, int k, int words, RnsConsts& C, const char* fn) {
  CKKS_REQUIRE(primes != nullptr && k >= 1 && k <= 8, "%s: 1..8 primes required", fn);
  CKKS_REQUIRE(words >= 1 && words <= 8, "%s: words outside [1, 8]", fn);
  C.k = k;
  C.words = words;
  int bits = 0;
  for (int i = 0; i < k; ++i) {
    const u64 p = primes[i];
    CKKS_REQUIRE(p >= 3 && p < (1ull << 62), "%s: prime %d outside [3, 2^62)", fn, i);
    for (int j = 0; j < i; ++j) CKKS_REQUIRE(primes[j] != p, "%s: primes must be distinct", fn);
    C.p[i] = p;
    C.r64[i] = h_twp((u64)(((unsigned __int128)1 << 64) % p), p);
    u64 pk = 1;
    for (int m = 0; m < i; ++m) {
      u64 pm = 1;
      for (int t = 0; t < m; ++t) pm = h_mulmod(pm, primes[t] % p, p);
      C.pmod[i][m] = h_twp(pm, p);
      pk = h_mulmod(pk, primes[m] % p, p);
    }
    C.pinv[i] = h_twp(i ? h_invmod(pk, p) : 1, p);
    bits += 64 - __builtin_clzll(p);
  }
  CKKS_REQUIRE(bits <= 64 * words, "%s: product of primes needs more than %d words", fn, words);
  u64 acc[8] = {1, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < k; ++i) {
    for (int w = 0; w < 8; ++w) C.pw[i][w] = w < words ? acc[w] : 0;
    mw_mul_small(acc, 8, primes[i]);
  }
  for (int w = 0; w < 8; ++w) C.mw[w] = acc[w];
  // (M - 1) / 2  (M odd)
  u64 h[8];
  for (int w = 0; w < 8; ++w) h[w] = acc[w];
  h[0] -= 1;
  for (int w = 0; w < 8; ++w) C.hw[w] = (h[w] >> 1) | (w + 1 < 8 ? (h[w + 1] << 63) : 0);
  return CKKS_OK;
}

extern "C" int ckks_rns_split(const uint64_t* primes, int n_primes, uint64_t* out,
                              const uint64_t* in, int64_t n, int words, int centered, void* stream) {
  RnsConsts C;
  if (int rc = make_rns(primes, n_primes, words, C, "ckks_rns_split")) return rc;
  if (n <= 0) return CKKS_OK;
  k_rns_split<<<grid1d((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), n, C, centered);
  return ckks_check_launch("ckks_rns_split");
}

extern "C" int ckks_rns_merge(const uint64_t* primes, int n_primes, uint64_t* out,
                              const uint64_t* in, int64_t n, int words, int centered, void* stream) {
  RnsConsts C;
  if (int rc = make_rns(primes, n_primes, words, C, "ckks_rns_merge")) return rc;
  if (n <= 0) return CKKS_OK;
  k_rns_merge<<<grid1d((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), n, C, centered);
  return ckks_check_launch("ckks_rns_merge");
}

// ---------------------------------------------------------------- gear controller
// rtl/m4/adaptive_gear_ctrl.sv:43-99 as a host-side state machine; energies
// and thresholds are 128-bit (the RTL accumulator is 106 bits).
static inline unsigned __int128 u128(uint64_t lo, uint64_t hi) {
  return ((unsigned __int128)hi << 64) | lo;
}

extern "C" int ckks_gear_ctrl_init(ckks_gear_ctrl* g, const uint64_t thresh_lo[3],
                                   const uint64_t thresh_hi[3], int hyst_cnt) {
  CKKS_REQUIRE(g != nullptr && thresh_lo != nullptr, "ckks_gear_ctrl_init: NULL argument");
  CKKS_REQUIRE(hyst_cnt >= 0, "ckks_gear_ctrl_init: hyst_cnt < 0");
  for (int i = 0; i < 3; ++i) {
    g->thresh_lo[i] = thresh_lo[i];
    g->thresh_hi[i] = thresh_hi ? thresh_hi[i] : 0;
  }
  g->hyst_cnt = hyst_cnt;
  g->gear = 3;
  g->counter = 0;
  g->candidate = 3;
  return CKKS_OK;
}

extern "C" int ckks_gear_ctrl_raw(const ckks_gear_ctrl* g, uint64_t energy_lo, uint64_t energy_hi) {
  const unsigned __int128 e = u128(energy_lo, energy_hi);
  if (e >= u128(g->thresh_lo[0], g->thresh_hi[0])) return 0;
  if (e >= u128(g->thresh_lo[1], g->thresh_hi[1])) return 1;
  if (e >= u128(g->thresh_lo[2], g->thresh_hi[2])) return 2;
  return 3;
}

extern "C" int ckks_gear_ctrl_flush(ckks_gear_ctrl* g, uint64_t energy_lo, uint64_t energy_hi,
                                    int hysteresis_en, int manual_en, int manual_gear) {
  if (!g) return ckks_set_error(CKKS_EINVAL, "ckks_gear_ctrl_flush: NULL state"), -1;
  const int raw = ckks_gear_ctrl_raw(g, energy_lo, energy_hi);
  if (manual_en) {
    g->gear = manual_gear;
    g->counter = 0;
    return manual_gear;
  }
  if (!hysteresis_en) {
    g->gear = raw;
    return g->gear;
  }
  if (raw > g->gear) {
    const int before = g->counter;
    if (raw == g->candidate) {
      g->counter += 1;
    } else {
      g->candidate = raw;
      g->counter = 1;
    }
    if (before >= g->hyst_cnt) {
      g->candidate = g->gear;
      g->gear = raw;
      g->counter = 0;
    }
  } else if (raw < g->gear) {
    g->gear = raw;
    g->counter = 0;
    g->candidate = raw;
  } else {
    g->counter = 0;
    g->candidate = raw;
  }
  return g->gear;
}
