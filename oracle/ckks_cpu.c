/*
 * ckks_cpu.c - native CPU restatement of the RNS ct-mult + relinearisation +
 * rescale (test infrastructure: the timed CPU baseline and a second oracle).
 *
 * The same algorithm, value for value, as oracle/rns_ckks.py
 * ct_mul_relin_rescale (which states it from the CKKS mathematics; the
 * reference has no RNS keyswitch or rescale, only the single-modulus
 * scripts/verify_keyswitch.py:62 relin and scripts/verify_rescale.py:38
 * rescale): per RNS limb tensor product, hybrid keyswitch with dnum = level
 * digits and one special prime (ModUp by a transform of each digit to every
 * prime, key inner product, ModDown by the centred special-prime part), and
 * the RNS rescale by the last limb.  Transforms are the merged negacyclic
 * Cooley-Tukey forward (twiddles psi^brv(k), bit-reversed evaluations out)
 * and its Gentleman-Sande inverse with N^-1, as oracle/ntt.py
 * merged_forward / merged_inverse.
 *
 * Arithmetic (moduli below 2^50): products by a fixed twiddle use Shoup's
 * precomputed quotient w' = floor(w 2^64 / q); products of two variables use
 * a floating-point quotient estimate (q_est = round(a b / q) in double
 * precision, r = a b - q_est q in wrapping 64-bit arithmetic, one correction),
 * exact because a b / q < 2^50 is estimated to within 1.
 *
 * Threads: pairs are split over `threads` POSIX threads.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ arithmetic */
static inline u64 shoup_pre(u64 w, u64 q) { return (u64)(((u128)w << 64) / q); }

static inline u64 mul_shoup(u64 x, u64 w, u64 ws, u64 q) {
  const u64 qe = (u64)(((u128)x * ws) >> 64);
  u64 r = x * w - qe * q;
  return r >= q ? r - q : r;
}

static inline u64 mulmod(u64 a, u64 b, u64 q, double qinv) {
  const u64 qe = (u64)((double)a * (double)b * qinv); /* floor of the estimate: off by at most one */
  int64_t r = (int64_t)(a * b - qe * q);
  if (r < 0) r += (int64_t)q;
  if (r >= (int64_t)q) r -= (int64_t)q;
  return (u64)r;
}

static inline u64 addmod(u64 a, u64 b, u64 q) {
  const u64 s = a + b;
  return s >= q ? s - q : s;
}
static inline u64 submod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + q - b; }

static u64 powmod(u64 b, u64 e, u64 q, double qinv) {
  u64 r = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) r = mulmod(r, b, q, qinv);
    b = mulmod(b, b, q, qinv);
    e >>= 1;
  }
  return r;
}
static u64 invmod(u64 a, u64 q, double qinv) { return powmod(a, q - 2, q, qinv); } /* q prime */

/* residue x mod q_from, centred to (-q_from/2, q_from/2], reduced mod q_to */
static inline u64 centred_to(u64 x, u64 q_from, u64 q_to) {
  if (x > q_from / 2) {
    const u64 m = (q_from - x) % q_to; /* |x - q_from| mod q_to */
    return m ? q_to - m : 0;
  }
  return x % q_to;
}

/* ------------------------------------------------------------------ transforms */
typedef struct {
  u64 q, ninv, ninv_s;
  double qinv;
  u64 *fw, *fws, *iw, *iws; /* [n]: psi^brv(k), psi^-brv(k) and their Shoup quotients */
} Prime;

static unsigned brv(unsigned k, int logn) {
  unsigned r = 0;
  for (int i = 0; i < logn; ++i) r |= ((k >> i) & 1u) << (logn - 1 - i);
  return r;
}

static int prime_init(Prime* P, u64 q, u64 psi, int logn) {
  const int n = 1 << logn;
  P->q = q;
  P->qinv = 1.0 / (double)q;
  P->fw = malloc(4 * (size_t)n * sizeof(u64));
  if (!P->fw) return -1;
  P->fws = P->fw + n;
  P->iw = P->fws + n;
  P->iws = P->iw + n;
  const u64 pinv = invmod(psi, q, P->qinv);
  P->fw[0] = P->iw[0] = 1;
  for (int k = 1; k < n; ++k) {
    const unsigned e = brv((unsigned)k, logn);
    P->fw[k] = powmod(psi, e, q, P->qinv);
    P->iw[k] = powmod(pinv, e, q, P->qinv);
  }
  for (int k = 0; k < n; ++k) {
    P->fws[k] = shoup_pre(P->fw[k], q);
    P->iws[k] = shoup_pre(P->iw[k], q);
  }
  P->ninv = invmod((u64)n % q, q, P->qinv);
  P->ninv_s = shoup_pre(P->ninv, q);
  return 0;
}

/* x w mod q up to one q: r in [0, 2q) for any x < 2^64 (Shoup, no correction) */
static inline u64 mul_shoup_lazy(u64 x, u64 w, u64 ws, u64 q) {
  const u64 qe = (u64)(((u128)x * ws) >> 64);
  return x * w - qe * q;
}

/* merged forward: natural coefficients in [0, q) -> bit-reversed evaluations
 * in [0, q).  Harvey's lazy butterflies: values stay in [0, 4q) between
 * stages (q < 2^50, so 4q fits easily), one final reduction. */
static void ntt_fwd(u64* x, const Prime* P, int n) {
  const u64 q = P->q, q2 = 2 * q;
  for (int m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1) {
    for (int i = 0; i < m; ++i) {
      const u64 w = P->fw[m + i], ws = P->fws[m + i];
      u64* a = x + 2 * (size_t)i * t;
      u64* b = a + t;
      for (int j = 0; j < t; ++j) {
        u64 u = a[j];
        u = u >= q2 ? u - q2 : u;
        const u64 v = mul_shoup_lazy(b[j], w, ws, q);
        a[j] = u + v;
        b[j] = u + q2 - v;
      }
    }
  }
  for (int j = 0; j < n; ++j) {
    u64 u = x[j];
    u = u >= q2 ? u - q2 : u;
    x[j] = u >= q ? u - q : u;
  }
}

/* Gentleman-Sande inverse of ntt_fwd, including N^-1: inputs in [0, q),
 * values in [0, 2q) between stages, outputs in [0, q) */
static void ntt_inv(u64* x, const Prime* P, int n) {
  const u64 q = P->q, q2 = 2 * q;
  for (int m = n >> 1, t = 1; m >= 1; m >>= 1, t <<= 1) {
    for (int i = 0; i < m; ++i) {
      const u64 w = P->iw[m + i], ws = P->iws[m + i];
      u64* a = x + 2 * (size_t)i * t;
      u64* b = a + t;
      for (int j = 0; j < t; ++j) {
        const u64 u = a[j], v = b[j];
        const u64 s = u + v;
        a[j] = s >= q2 ? s - q2 : s;
        b[j] = mul_shoup_lazy(u + q2 - v, w, ws, q);
      }
    }
  }
  for (int j = 0; j < n; ++j) x[j] = mul_shoup(x[j], P->ninv, P->ninv_s, q);
}

/* ------------------------------------------------------------------ ct-mult */
typedef struct {
  int logn, n, nq;        /* nq: q-primes of the key basis (its special prime last) */
  Prime* pr;              /* [nq + 1] */
  u64* pinv;              /* [nq]: p^-1 mod q_i */
  u64* qtinv;             /* [nq][nq]: q_t^-1 mod q_i */
} cc_ctx;

void cc_destroy(cc_ctx* c) {
  if (!c) return;
  if (c->pr)
    for (int i = 0; i <= c->nq; ++i) free(c->pr[i].fw);
  free(c->pr);
  free(c->pinv);
  free(c->qtinv);
  free(c);
}

/* primes: nq q-primes then the special prime; psi: a primitive 2N-th root of
 * unity of each (the oracle's root_2n); every prime below 2^50.  NULL on
 * failure. */
cc_ctx* cc_create(int logn, int nq, const u64* primes, const u64* psi) {
  if (logn < 1 || logn > 17 || nq < 1 || nq > 62) return NULL;
  for (int i = 0; i <= nq; ++i)
    if (primes[i] < 3 || primes[i] >= (1ull << 50)) return NULL;
  cc_ctx* c = calloc(1, sizeof(cc_ctx));
  if (!c) return NULL;
  c->logn = logn;
  c->n = 1 << logn;
  c->nq = nq;
  c->pr = calloc((size_t)nq + 1, sizeof(Prime));
  c->pinv = malloc((size_t)nq * sizeof(u64));
  c->qtinv = malloc((size_t)nq * nq * sizeof(u64));
  if (!c->pr || !c->pinv || !c->qtinv) {
    cc_destroy(c);
    return NULL;
  }
  for (int i = 0; i <= nq; ++i)
    if (prime_init(&c->pr[i], primes[i], psi[i], logn)) {
      cc_destroy(c);
      return NULL;
    }
  const u64 p = primes[nq];
  for (int i = 0; i < nq; ++i) {
    const Prime* P = &c->pr[i];
    c->pinv[i] = invmod(p % P->q, P->q, P->qinv);
    for (int t = 0; t < nq; ++t) c->qtinv[(size_t)t * nq + i] = t == i ? 0 : invmod(primes[t] % P->q, P->q, P->qinv);
  }
  return c;
}

/* One pair: a, b [2][l][N] evaluation domain; ksk [nq][2][nq + 1][N];
 * out [2][l - 1][N].  w: 10 l N + 4 N words of workspace. */
static void ct_mul_one(const cc_ctx* c, u64* out, const u64* a, const u64* b, const u64* ksk, int l, u64* w) {
  const int n = c->n, nq = c->nq;
  const size_t LN = (size_t)l * n;
  u64* d0 = w;              /* [l][N] */
  u64* d1 = d0 + LN;        /* [l][N] */
  u64* d2 = d1 + LN;        /* [l][N] evaluation */
  u64* d2c = d2 + LN;       /* [l][N] coefficient digits */
  u64* acc = d2c + LN;      /* [2][l + 1][N] */
  u64* tmp = acc + 2 * (LN + n); /* [N] */
  u64* full = tmp + n;      /* [2][l][N] */
  /* tensor product per limb */
  for (int i = 0; i < l; ++i) {
    const Prime* P = &c->pr[i];
    const u64 q = P->q;
    const u64 *a0 = a + (size_t)i * n, *a1 = a + LN + (size_t)i * n;
    const u64 *b0 = b + (size_t)i * n, *b1 = b + LN + (size_t)i * n;
    for (int j = 0; j < n; ++j) {
      d0[(size_t)i * n + j] = mulmod(a0[j], b0[j], q, P->qinv);
      d1[(size_t)i * n + j] = addmod(mulmod(a0[j], b1[j], q, P->qinv), mulmod(a1[j], b0[j], q, P->qinv), q);
      d2[(size_t)i * n + j] = mulmod(a1[j], b1[j], q, P->qinv);
    }
  }
  /* digits: d2 in the coefficient domain */
  memcpy(d2c, d2, LN * sizeof(u64));
  for (int j = 0; j < l; ++j) ntt_inv(d2c + (size_t)j * n, &c->pr[j], n);
  /* ModUp + key inner product: target r < l is q_r (key limb r), r = l the special prime (key limb nq) */
  memset(acc, 0, 2 * (LN + n) * sizeof(u64));
  for (int r = 0; r <= l; ++r) {
    const int pidx = r < l ? r : nq, kl = pidx;
    const Prime* P = &c->pr[pidx];
    const u64 q = P->q;
    for (int j = 0; j < l; ++j) {
      const u64* dj;
      if (r == j) {
        dj = d2 + (size_t)j * n;
      } else {
        for (int e = 0; e < n; ++e) tmp[e] = d2c[(size_t)j * n + e] % q;
        ntt_fwd(tmp, P, n);
        dj = tmp;
      }
      for (int k = 0; k < 2; ++k) {
        const u64* kv = ksk + (((size_t)j * 2 + k) * (nq + 1) + kl) * n;
        u64* ac = acc + ((size_t)k * (l + 1) + r) * n;
        for (int e = 0; e < n; ++e) ac[e] = addmod(ac[e], mulmod(dj[e], kv[e], q, P->qinv), q);
      }
    }
  }
  /* ModDown by p, then add d0 / d1 */
  const Prime* PP = &c->pr[nq];
  for (int k = 0; k < 2; ++k) {
    u64* accp = acc + ((size_t)k * (l + 1) + l) * n;
    ntt_inv(accp, PP, n);
    for (int i = 0; i < l; ++i) {
      const Prime* P = &c->pr[i];
      const u64 q = P->q;
      for (int e = 0; e < n; ++e) tmp[e] = centred_to(accp[e], PP->q, q);
      ntt_fwd(tmp, P, n);
      const u64* ai = acc + ((size_t)k * (l + 1) + i) * n;
      const u64* dk = (k ? d1 : d0) + (size_t)i * n;
      u64* f = full + ((size_t)k * l + i) * n;
      for (int e = 0; e < n; ++e) f[e] = addmod(dk[e], mulmod(submod(ai[e], tmp[e], q), c->pinv[i], q, P->qinv), q);
    }
  }
  /* rescale by q_t, t = l - 1 */
  const int t = l - 1;
  const Prime* PT = &c->pr[t];
  for (int k = 0; k < 2; ++k) {
    u64* ft = full + ((size_t)k * l + t) * n;
    ntt_inv(ft, PT, n);
    for (int i = 0; i < t; ++i) {
      const Prime* P = &c->pr[i];
      const u64 q = P->q;
      for (int e = 0; e < n; ++e) tmp[e] = centred_to(ft[e], PT->q, q);
      ntt_fwd(tmp, P, n);
      const u64* fi = full + ((size_t)k * l + i) * n;
      u64* o = out + ((size_t)k * t + i) * n;
      const u64 ci = c->qtinv[(size_t)t * nq + i];
      for (int e = 0; e < n; ++e) o[e] = mulmod(submod(fi[e], tmp[e], q), ci, q, P->qinv);
    }
  }
}

typedef struct {
  const cc_ctx* c;
  u64* out;
  const u64 *a, *b, *ksk;
  int l;
  long long lo, hi;
  int rc;
} Job;

static void* run_job(void* arg) {
  Job* J = (Job*)arg;
  const cc_ctx* c = J->c;
  const size_t in_ct = 2 * (size_t)J->l * c->n, out_ct = 2 * (size_t)(J->l - 1) * c->n;
  u64* w = malloc((10 * (size_t)J->l * c->n + 4 * (size_t)c->n) * sizeof(u64));
  if (!w) {
    J->rc = -1;
    return NULL;
  }
  for (long long i = J->lo; i < J->hi; ++i)
    ct_mul_one(c, J->out + i * out_ct, J->a + i * in_ct, J->b + i * in_ct, J->ksk, J->l, w);
  free(w);
  J->rc = 0;
  return NULL;
}

/* n_ct pairs, ciphertexts [n_ct][2][level][N] (evaluation domain), key
 * [nq][2][nq + 1][N], out [n_ct][2][level - 1][N]; 0 on success. */
int cc_ct_mul_relin_rescale(const cc_ctx* c, u64* out, const u64* a, const u64* b, const u64* ksk, long long n_ct,
                            int level, int threads) {
  if (!c || level < 2 || level > c->nq || n_ct < 0) return -1;
  if (n_ct == 0) return 0;
  if (threads < 1) threads = 1;
  if (threads > n_ct) threads = (int)n_ct;
  Job* jobs = calloc((size_t)threads, sizeof(Job));
  pthread_t* th = calloc((size_t)threads, sizeof(pthread_t));
  if (!jobs || !th) {
    free(jobs);
    free(th);
    return -1;
  }
  int rc = 0;
  for (int t = 0; t < threads; ++t) {
    jobs[t] = (Job){c, out, a, b, ksk, level, n_ct * t / threads, n_ct * (t + 1) / threads, 0};
    if (t && pthread_create(&th[t], NULL, run_job, &jobs[t])) {
      jobs[t].rc = -1;
      th[t] = 0;
    }
  }
  run_job(&jobs[0]);
  for (int t = 1; t < threads; ++t)
    if (th[t]) pthread_join(th[t], NULL);
  for (int t = 0; t < threads; ++t) rc |= jobs[t].rc;
  free(jobs);
  free(th);
  return rc ? -1 : 0;
}
