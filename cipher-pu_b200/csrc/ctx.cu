// ctx.cu - context creation (prime constants, twiddle tables) and the
// thread-local error channel of the C ABI.
#include <cstring>
#include <mutex>

#include "ctx.hpp"

static thread_local std::string g_last_error;

int ckks_set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int ckks_check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return ckks_set_error(CKKS_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return CKKS_OK;
}

extern "C" int ckks_abi_version(void) { return 1; }

extern "C" const char* ckks_last_error(void) { return g_last_error.c_str(); }

static int bitrev(int i, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) {
    r = (r << 1) | (i & 1);
    i >>= 1;
  }
  return r;
}

static bool is_prime_u64(u64 n) {
  if (n < 2) return false;
  static const u64 bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  for (u64 p : bases)
    if (n % p == 0) return n == p;
  u64 d = n - 1;
  int s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    ++s;
  }
  for (u64 a : bases) {
    u64 x = h_powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; ++r) {
      x = h_mulmod(x, x, n);
      if (x == n - 1) {
        comp = false;
        break;
      }
    }
    if (comp) return false;
  }
  return true;
}

// root^e mod q for e in [0, n)
static std::vector<u64> h_powers(u64 root, int n, u64 q) {
  std::vector<u64> p(n);
  u64 cur = 1 % q;
  for (int e = 0; e < n; ++e) {
    p[e] = cur;
    cur = h_mulmod(cur, root, q);
  }
  return p;
}

// First stage of the last register pass of an N = 2^log_n transform with
// 2^k coefficients per thread (the pass split of NttShape in ntt.cuh).
static int last_pass_s0(int log_n, int k) {
  k = k < log_n ? k : log_n;
  const int r = log_n - k;
  if (r == 0) return 0;
  const int np = (r + k - 1) / k;
  const int kp_last = r / np + ((np - 1) < (r % np) ? 1 : 0);
  return log_n - kp_last;
}

// Forward table: group ii of stage m = 2^s at m + ii, except in the stages
// s >= s0 of the last pass, where ii = block * 2^u + grp (u = s - s0) goes to
// m + grp * 2^s0 + block.
template <typename F>
static void fill_fwd(TwD* dst, int log_n, int s0, F&& value, u64 q) {
  for (int s = 0; s < log_n; ++s) {
    const int m = 1 << s;
    const int u = s - s0;
    for (int ii = 0; ii < m; ++ii) {
      const int at = u >= 0 ? m + (ii & ((1 << u) - 1)) * (1 << s0) + (ii >> u) : m + ii;
      dst[at] = h_twd(value(m, ii), q);
    }
  }
}

// Inverse table: stage s (h = N / 2^(s+1)) holds w^(k 2^s), k < h, at h + k;
// pw[e] = w^e.
static void fill_inv(TwD* dst, int log_n, const std::vector<u64>& pw, u64 q) {
  const int n = 1 << log_n;
  for (int s = 0; s < log_n; ++s) {
    const int h = n >> (s + 1);
    for (int k = 0; k < h; ++k) dst[h + k] = h_twd(pw[(size_t)k << s], q);
  }
}

static void free_ctx(ckks_ctx* c) {
  if (!c) return;
  cudaFree(c->d_pi);
  cudaFree(c->d_tw);
  cudaFree(c->d_pinv);
  cudaFree(c->d_qtinv);
  cudaFree(c->d_ntt_tc);
  delete c;
}

extern "C" int ckks_ctx_create(int log_n, int n_primes, int n_special, const uint64_t* primes,
                               const uint64_t* psi, const uint64_t* omega, ckks_ctx** out) {
  CKKS_REQUIRE(out != nullptr, "ckks_ctx_create: out is NULL");
  *out = nullptr;
  CKKS_REQUIRE(log_n >= 1 && log_n <= 14, "ckks_ctx_create: log_n=%d outside [1, 14]", log_n);
  CKKS_REQUIRE(n_primes >= 1 && n_primes <= 64, "ckks_ctx_create: n_primes=%d outside [1, 64]",
               n_primes);
  CKKS_REQUIRE(n_special >= 0 && n_special <= 1 && n_special < n_primes,
               "ckks_ctx_create: n_special=%d (must be 0 or 1 and < n_primes)", n_special);
  CKKS_REQUIRE(primes != nullptr && psi != nullptr, "ckks_ctx_create: NULL primes/psi");
  const int n = 1 << log_n;
  ckks_ctx* c = new ckks_ctx();
  c->log_n = log_n;
  c->n = n;
  c->n_primes = n_primes;
  c->n_special = n_special;
  c->n_q = n_primes - n_special;
  cudaGetDevice(&c->device);
  std::vector<TwD> tw((size_t)n_primes * TWF_SLOTS * n);
  for (int i = 0; i < n_primes; ++i) {
    const u64 q = primes[i];
    if (q < 3 || q >= (1ull << 47) || !is_prime_u64(q)) {
      free_ctx(c);
      return ckks_set_error(CKKS_EINVAL, "ckks_ctx_create: primes[%d]=%llu is not a prime in [3, 2^47)",
                            i, (unsigned long long)q);
    }
    if ((q - 1) % (u64)n != 0) {
      free_ctx(c);
      return ckks_set_error(CKKS_EINVAL, "ckks_ctx_create: N=%d does not divide primes[%d]-1", n, i);
    }
    u64 ps = psi[i] % q;
    bool nega = ps != 0;
    if (nega) {
      if (h_powmod(ps, (u64)n, q) != q - 1) {
        free_ctx(c);
        return ckks_set_error(CKKS_EINVAL, "ckks_ctx_create: psi[%d] is not a primitive 2N-th root", i);
      }
    }
    u64 om = (omega && omega[i]) ? omega[i] % q : (nega ? h_mulmod(ps, ps, q) : 0);
    if (om == 0 || h_powmod(om, (u64)n, q) != 1 || (n > 1 && h_powmod(om, (u64)n / 2, q) == 1)) {
      free_ctx(c);
      return ckks_set_error(CKKS_EINVAL, "ckks_ctx_create: omega[%d] is not a primitive N-th root", i);
    }
    c->primes.push_back(q);
    c->psi.push_back(ps);
    c->omega.push_back(om);
    c->has_nega.push_back(nega ? 1 : 0);
    PrimeInfo P;
    std::memset(&P, 0, sizeof(P));
    P.q = q;
    P.q2 = 2 * q;
    P.qlazy = q << 5;
    u64 inv = 1;  // q^{-1} mod 2^64 by Newton
    for (int k = 0; k < 7; ++k) inv *= 2 - q * inv;
    P.mont_qinv = (u64)0 - inv;
    P.r_mod = (u64)(((unsigned __int128)1 << 64) % q);
    P.r_mod_s = h_shoup(P.r_mod, q);
    P.one_s = h_shoup(1, q);
    P.ninv = h_invmod((u64)n % q, q);
    P.ninv_s = h_shoup(P.ninv, q);
    P.half = (q - 1) / 2;
    P.qd = (double)q;
    P.qinv_d = 1.0 / (double)q;
    c->h_pi.push_back(P);
    TwD* t = tw.data() + (size_t)i * TWF_SLOTS * n;
    for (int k = 0; k < TWF_SLOTS * n; ++k) t[k] = TwD{0.0, 0.0};
    const u64 ninv_q = h_invmod((u64)n % q, q);
    const u64 oinv = h_invmod(om, q);
    if (nega) {
      const std::vector<u64> pp = h_powers(ps, n, q);
      for (int k = 2; k <= 5; ++k)
        fill_fwd(t + (TWF_FWD2 + k - 2) * n, log_n, last_pass_s0(log_n, k), [&](int m, int ii) {
          return pp[bitrev(m + ii, log_n)];
        }, q);
      const u64 pinv = h_invmod(ps, q);
      fill_inv(t + TWF_INV * n, log_n, h_powers(h_mulmod(pinv, pinv, q), n, q), q);
      u64 cur = ninv_q;
      for (int j = 0; j < n; ++j) {
        t[TWF_POST * n + j] = h_twd(cur, q);
        cur = h_mulmod(cur, pinv, q);
      }
    }
    const std::vector<u64> po = h_powers(om, n, q);
    auto cyc_tw = [&](int m, int ii) { return po[(bitrev(m + ii, log_n) - n / (2 * m)) / 2]; };
    for (int k = 2; k <= 5; ++k) fill_fwd(t + (TWF_FWDC2 + k - 2) * n, log_n, last_pass_s0(log_n, k), cyc_tw, q);
    fill_inv(t + TWF_INV_CYC * n, log_n, h_powers(oinv, n, q), q);
    for (int j = 0; j < n; ++j) t[TWF_POST_CYC * n + j] = h_twd(ninv_q, q);
  }
  // keyswitch / rescale constants
  const int nq = c->n_q;
  std::vector<TwPair> pinv(nq), qtinv((size_t)nq * nq);
  c->h_pinv.assign(nq, 0);
  c->h_qtinv.assign(nq, std::vector<u64>(nq, 0));
  for (int i = 0; i < nq; ++i) {
    TwPair z;
    z.w = 0;
    z.ws = 0;
    pinv[i] = z;
    if (n_special) {
      const u64 p = c->primes[nq];
      const u64 v = h_invmod(p % c->primes[i], c->primes[i]);
      pinv[i] = h_twp(v, c->primes[i]);
      c->h_pinv[i] = v;
    }
  }
  for (int t = 0; t < nq; ++t)
    for (int i = 0; i < nq; ++i) {
      TwPair z;
      z.w = 0;
      z.ws = 0;
      qtinv[(size_t)t * nq + i] = z;
      if (i < t && c->primes[t] % c->primes[i] != 0) {
        const u64 v = h_invmod(c->primes[t] % c->primes[i], c->primes[i]);
        qtinv[(size_t)t * nq + i] = h_twp(v, c->primes[i]);
        c->h_qtinv[t][i] = v;
      }
    }
  cudaError_t e = cudaSuccess;
  e = cudaMalloc(&c->d_pi, sizeof(PrimeInfo) * n_primes);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_tw, sizeof(TwD) * tw.size());
  if (e == cudaSuccess) e = cudaMalloc(&c->d_pinv, sizeof(TwPair) * nq);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_qtinv, sizeof(TwPair) * (size_t)nq * nq);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_pi, c->h_pi.data(), sizeof(PrimeInfo) * n_primes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_tw, tw.data(), sizeof(TwD) * tw.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_pinv, pinv.data(), sizeof(TwPair) * nq, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_qtinv, qtinv.data(), sizeof(TwPair) * (size_t)nq * nq,
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    free_ctx(c);
    return ckks_set_error(CKKS_ECUDA, "ckks_ctx_create: %s", cudaGetErrorString(e));
  }
  *out = c;
  return CKKS_OK;
}

namespace {
// smallest generator of (Z/qZ)^* (q prime): q - 1 = 2^k m with m < 2^47, its
// distinct prime factors by trial division, then the first g with
// g^((q-1)/f) != 1 for every factor f
u64 smallest_generator(u64 q) {
  std::vector<u64> fs;
  u64 m = q - 1;
  for (u64 d = 2; d * d <= m; d += (d == 2 ? 1 : 2))
    if (m % d == 0) {
      fs.push_back(d);
      while (m % d == 0) m /= d;
    }
  if (m > 1) fs.push_back(m);
  for (u64 g = 2;; ++g) {
    bool ok = true;
    for (u64 f : fs) ok = ok && h_powmod(g, (q - 1) / f, q) != 1;
    if (ok) return g;
  }
}
}  // namespace

extern "C" int ckks_ctx_create_params(const ckks_params* p, ckks_ctx** out) {
  const char* fn = "ckks_ctx_create_params";
  CKKS_REQUIRE(p != nullptr && out != nullptr, "%s: NULL argument", fn);
  *out = nullptr;
  CKKS_REQUIRE(p->reserved == 0, "%s: reserved field must be 0", fn);
  CKKS_REQUIRE(p->log_n >= 1 && p->log_n <= 14, "%s: log_n=%d outside [1, 14]", fn, p->log_n);
  CKKS_REQUIRE(p->n_primes >= 1 && p->n_primes <= 64, "%s: n_primes=%d outside [1, 64]", fn, p->n_primes);
  CKKS_REQUIRE(p->primes != nullptr, "%s: primes is NULL", fn);
  const u64 n = 1ull << p->log_n;
  std::vector<uint64_t> psi(p->n_primes), om(p->n_primes);
  for (int i = 0; i < p->n_primes; ++i) {
    const u64 q = p->primes[i];
    CKKS_REQUIRE(q >= 3 && q < (1ull << 47) && is_prime_u64(q), "%s: primes[%d]=%llu is not a prime in [3, 2^47)",
                 fn, i, (unsigned long long)q);
    CKKS_REQUIRE((q - 1) % n == 0, "%s: N=%llu does not divide primes[%d]-1", fn, (unsigned long long)n, i);
    u64 g = 0;
    if (p->psi && p->psi[i]) {
      psi[i] = p->psi[i];
    } else if ((q - 1) % (2 * n) == 0) {
      g = smallest_generator(q);
      psi[i] = h_powmod(g, (q - 1) / (2 * n), q);
    } else {
      psi[i] = 0;
    }
    if (p->omega && p->omega[i]) {
      om[i] = p->omega[i];
    } else if (psi[i]) {
      om[i] = h_mulmod(psi[i], psi[i], q);
    } else {
      if (!g) g = smallest_generator(q);
      om[i] = h_powmod(g, (q - 1) / n, q);
    }
  }
  ckks_ctx* c = nullptr;
  if (int rc = ckks_ctx_create(p->log_n, p->n_primes, p->n_special, p->primes, psi.data(), om.data(), &c)) return rc;
  c->scale = p->scale;
  c->sigma = p->sigma;
  c->seed = p->seed;
  *out = c;
  return CKKS_OK;
}

extern "C" int ckks_ctx_get_params(const ckks_ctx* ctx, ckks_params* out) {
  CKKS_REQUIRE(ctx != nullptr && out != nullptr, "ckks_ctx_get_params: NULL argument");
  out->log_n = ctx->log_n;
  out->n_primes = ctx->n_primes;
  out->n_special = ctx->n_special;
  out->reserved = 0;
  out->primes = reinterpret_cast<const uint64_t*>(ctx->primes.data());
  out->psi = reinterpret_cast<const uint64_t*>(ctx->psi.data());
  out->omega = reinterpret_cast<const uint64_t*>(ctx->omega.data());
  out->scale = ctx->scale;
  out->sigma = ctx->sigma;
  out->seed = ctx->seed;
  return CKKS_OK;
}

extern "C" int ckks_ctx_destroy(ckks_ctx* ctx) {
  free_ctx(ctx);
  return CKKS_OK;
}

extern "C" int ckks_ctx_set_tuning(ckks_ctx* ctx, int param, int value) {
  CKKS_REQUIRE(ctx != nullptr, "ckks_ctx_set_tuning: ctx is NULL");
  switch (param) {
    case CKKS_TUNE_CM_LOG_ELEMS:
      CKKS_REQUIRE(value == 0 || (value >= 2 && value <= 5),
                   "ckks_ctx_set_tuning: ct-mult log2 elements per thread must be 0 or in [2, 5]");
      ctx->tune_cm_k = value;
      return CKKS_OK;
    case CKKS_TUNE_CM_MIN_BLOCKS:
      CKKS_REQUIRE(value == 0 || value == 1 || value == 2,
                   "ckks_ctx_set_tuning: ct-mult register budget must be 0, 1 (balanced) or 2 (tight)");
      ctx->tune_cm_minb = value;
      return CKKS_OK;
    case CKKS_TUNE_NTT_LOG_ELEMS:
      CKKS_REQUIRE(value == 0 || (value >= 2 && value <= 5),
                   "ckks_ctx_set_tuning: transform log2 elements per thread must be 0 or in [2, 5]");
      ctx->tune_ntt_k = value;
      return CKKS_OK;
    case CKKS_TUNE_CM_UNITS_PER_CTA:
      CKKS_REQUIRE(value >= 0 && value <= 8,
                   "ckks_ctx_set_tuning: ct-mult work units per CTA must be in [0, 8]");
      ctx->tune_cm_upc = value;
      return CKKS_OK;
    case CKKS_TUNE_CM_TENSOR_TMA:
      CKKS_REQUIRE(value >= 0 && value <= 2,
                   "ckks_ctx_set_tuning: ct-mult tensor variant must be 0, 1 (TMA-fed) or 2 (one CTA per unit)");
      ctx->tune_cm_tma = value;
      return CKKS_OK;
    case CKKS_TUNE_CM_SPLIT:
      CKKS_REQUIRE(value >= 0 && value <= 16,
                   "ckks_ctx_set_tuning: ct-mult sub-batches must be in [0, 16]");
      ctx->tune_cm_split = value;
      return CKKS_OK;
    case CKKS_TUNE_CM_FUSED:
      CKKS_REQUIRE(value >= 0 && value <= 2,
                   "ckks_ctx_set_tuning: ct-mult path must be 0 (auto), 1 (fused) or 2 (three kernels)");
      ctx->tune_cm_fused = value;
      return CKKS_OK;
    case CKKS_TUNE_CM_MODUP_TMEM:
      CKKS_REQUIRE(value >= 0 && value <= 2,
                   "ckks_ctx_set_tuning: ModUp accumulators must be 0 (auto), 1 (TMEM) or 2 (shared memory)");
      ctx->tune_cm_tmem = value;
      return CKKS_OK;
    case CKKS_TUNE_WAIT_CYCLES:
      CKKS_REQUIRE(value >= 0, "ckks_ctx_set_tuning: wait limit must be >= 0 SM cycles");
      ctx->tune_wait_cycles = value;
      return CKKS_OK;
    default:
      return ckks_set_error(CKKS_EINVAL, "ckks_ctx_set_tuning: unknown parameter %d", param);
  }
}
