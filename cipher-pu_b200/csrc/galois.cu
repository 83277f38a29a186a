// galois.cu - ring automorphisms psi_nu(f)(X) = f(X^nu) mod (X^N + 1) and
// multiplication by a monomial X^nu, per RNS limb.
//
// Coefficient domain: coefficient k of f lands on j = nu k mod N with sign
// (-1)^floor(nu k / N).  For odd nu that is a signed permutation (one gather
// per output word, k = j nu^-1 mod N); for even nu several k share one j and
// the terms are summed (atomic accumulation of non-negative representatives,
// then one reduction pass), which is the reference's definition for every nu.
// Evaluation domain (odd nu): slot i of the merged forward transform holds
// f(psi^(2 brv(i) + 1)), so psi_nu(f) at slot i is f at slot i' with
// 2 brv(i') + 1 = nu (2 brv(i) + 1) mod 2N: a pure permutation.
#include "dispatch.cuh"

__device__ __forceinline__ u64 neg_if(u64 x, bool neg, u64 q) { return (neg && x) ? q - x : x; }

// odd nu: out[j] = +-in[k], k = j * nuinv mod N
__global__ void k_automorph_odd(u64* __restrict__ out, const u64* __restrict__ in, long long total,
                                int log_n, int n_limbs, int prime_begin, u64 nu2n, u64 nuinv,
                                const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const u64 n = 1ull << log_n;
  const u64 j = (u64)idx & (n - 1);
  const long long row = idx >> log_n;
  const u64 q = pi[prime_begin + (int)(row % n_limbs)].q;
  const u64 k = (j * nuinv) & (n - 1);
  const u64 p = (nu2n * k) & (2 * n - 1);  // nu k mod 2N: (p mod N) == j
  out[idx] = neg_if(in[(size_t)row * n + k], p >= n, q);
}

// any nu: accumulate +-in[k] into out[nu k mod N] (out zeroed first)
__global__ void k_automorph_scatter(u64* __restrict__ out, const u64* __restrict__ in, long long total,
                                    int log_n, int n_limbs, int prime_begin, u64 nu2n,
                                    const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const u64 n = 1ull << log_n;
  const u64 k = (u64)idx & (n - 1);
  const long long row = idx >> log_n;
  const u64 q = pi[prime_begin + (int)(row % n_limbs)].q;
  const u64 p = (nu2n * k) & (2 * n - 1);
  const u64 v = neg_if(in[idx], p >= n, q);
  if (v) atomicAdd(out + (size_t)row * n + (p & (n - 1)), v);
}

// reduce the accumulated sums (each below N q < 2^61) to [0, q)
__global__ void k_reduce_rows(u64* __restrict__ x, long long total, int log_n, int n_limbs,
                              int prime_begin, const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const PrimeInfo P = pi[prime_begin + (int)((idx >> log_n) % n_limbs)];
  x[idx] = reduce_any(x[idx], P);
}

__global__ void k_automorph_eval(u64* __restrict__ out, const u64* __restrict__ in, long long total,
                                 int log_n, u64 nu2n) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const u64 n = 1ull << log_n;
  const long long row = idx >> log_n;
  out[idx] = in[(size_t)row * n + galois_eval_src((u64)idx & (n - 1), log_n, nu2n)];
}

// out[(k + nu) mod N] = +-in[k], sign flipped where k + nu mod 2N >= N
__global__ void k_monomial(u64* __restrict__ out, const u64* __restrict__ in, long long total, int log_n,
                           int n_limbs, int prime_begin, u64 nu2n, const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const u64 n = 1ull << log_n;
  const u64 k = (u64)idx & (n - 1);
  const long long row = idx >> log_n;
  const u64 q = pi[prime_begin + (int)(row % n_limbs)].q;
  const u64 p = (k + nu2n) & (2 * n - 1);
  out[(size_t)row * n + (p & (n - 1))] = neg_if(in[idx], p >= n, q);
}

static u64 inv_mod_pow2(u64 a, int bits) {  // a odd
  u64 x = 1;
  for (int i = 0; i < 7; ++i) x *= 2 - a * x;
  return bits >= 64 ? x : (x & ((1ull << bits) - 1));
}

static int check_rows(const ckks_ctx* ctx, const void* out, const void* in, int n_polys, int prime_begin,
                      int n_limbs, const char* fn) {
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_polys >= 0, "%s: n_polys < 0", fn);
  CKKS_REQUIRE(n_limbs >= 1 && prime_begin >= 0 && prime_begin + n_limbs <= ctx->n_primes,
               "%s: limb range [%d, %d) outside the %d context primes", fn, prime_begin,
               prime_begin + n_limbs, ctx->n_primes);
  CKKS_REQUIRE(n_polys == 0 || (out && in), "%s: NULL pointer argument", fn);
  CKKS_REQUIRE(n_polys == 0 || out != in, "%s: out must differ from in", fn);
  return CKKS_OK;
}

extern "C" int ckks_automorphism(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_polys,
                                 int prime_begin, int n_limbs, uint64_t nu, int eval_domain,
                                 void* stream) {
  const char* fn = "ckks_automorphism";
  if (int rc = check_rows(ctx, out, in, n_polys, prime_begin, n_limbs, fn)) return rc;
  const u64 n = (u64)ctx->n;
  const u64 nu2n = nu & (2 * n - 1);
  const long long total = (long long)n_polys * n_limbs * (long long)n;
  if (eval_domain) {
    CKKS_REQUIRE(nu2n & 1, "%s: the evaluation-domain automorphism needs an odd nu", fn);
    for (int l = 0; l < n_limbs; ++l)
      CKKS_REQUIRE(ctx->has_nega[prime_begin + l], "%s: prime %d has no 2N-th root", fn,
                   prime_begin + l);
  }
  if (total == 0) return CKKS_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned grid = grid1d((total + 255) / 256);
  if (eval_domain) {
    k_automorph_eval<<<grid, 256, 0, st>>>(reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in),
                                           total, ctx->log_n, nu2n);
  } else if (nu2n & 1) {
    k_automorph_odd<<<grid, 256, 0, st>>>(reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in),
                                          total, ctx->log_n, n_limbs, prime_begin, nu2n,
                                          inv_mod_pow2(nu2n, ctx->log_n), ctx->d_pi);
  } else {
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)total * sizeof(u64), st);
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    k_automorph_scatter<<<grid, 256, 0, st>>>(reinterpret_cast<u64*>(out),
                                              reinterpret_cast<const u64*>(in), total, ctx->log_n,
                                              n_limbs, prime_begin, nu2n, ctx->d_pi);
    if (int rc = ckks_check_launch(fn)) return rc;
    k_reduce_rows<<<grid, 256, 0, st>>>(reinterpret_cast<u64*>(out), total, ctx->log_n, n_limbs,
                                        prime_begin, ctx->d_pi);
  }
  return ckks_check_launch(fn);
}

extern "C" int ckks_mul_monomial(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_polys,
                                 int prime_begin, int n_limbs, uint64_t nu, void* stream) {
  const char* fn = "ckks_mul_monomial";
  if (int rc = check_rows(ctx, out, in, n_polys, prime_begin, n_limbs, fn)) return rc;
  const u64 n = (u64)ctx->n;
  const long long total = (long long)n_polys * n_limbs * (long long)n;
  if (total == 0) return CKKS_OK;
  k_monomial<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), total, ctx->log_n, n_limbs,
      prime_begin, nu & (2 * n - 1), ctx->d_pi);
  return ckks_check_launch(fn);
}
