// arith.cu - elementwise ciphertext arithmetic over all limbs of a level:
// ct + ct / ct - ct, ct x integer constant, ct + integer constant.  The
// building blocks of polynomial evaluation (activation approximations) and
// of layer sums; every value stays a canonical residue.
#include "dispatch.cuh"

// [n_ct][2][level][N]: limb of word idx
__device__ __forceinline__ int ct_limb(long long idx, int log_n, int level) {
  return (int)((idx >> log_n) % level);
}

__global__ void k_ct_addsub(u64* __restrict__ out, const u64* __restrict__ a, const u64* __restrict__ b,
                            long long total, int log_n, int level, int subtract,
                            const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const u64 q = pi[ct_limb(idx, log_n, level)].q;
  out[idx] = subtract ? submod(a[idx], b[idx], q) : addmod(a[idx], b[idx], q);
}

// m_res[limb] = m mod q_limb with its Shoup companion (host-computed)
struct ConstRes {
  u64 w[64];
  u64 ws[64];
};

__global__ void k_ct_mul_const(u64* __restrict__ out, const u64* __restrict__ in, long long total,
                               int log_n, int level, ConstRes M, const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int l = ct_limb(idx, log_n, level);
  out[idx] = shoup(in[idx], M.w[l], M.ws[l], pi[l].q);
}

// adds c_res[limb] to every word of component 0 (the evaluation-domain image
// of the constant polynomial c is c at every slot)
__global__ void k_ct_add_const(u64* __restrict__ out, const u64* __restrict__ in, long long total,
                               int log_n, int level, ConstRes C, const PrimeInfo* __restrict__ pi) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int l = ct_limb(idx, log_n, level);
  const bool comp0 = ((idx >> log_n) / level) % 2 == 0;
  out[idx] = comp0 ? addmod(in[idx], C.w[l], pi[l].q) : in[idx];
}

static int check_ct(const ckks_ctx* ctx, int n_ct, int level, const char* fn) {
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_ct >= 0, "%s: n_ct < 0", fn);
  CKKS_REQUIRE(level >= 1 && level <= ctx->n_primes && level <= 64, "%s: level=%d outside [1, %d]", fn,
               level, ctx->n_primes < 64 ? ctx->n_primes : 64);
  return CKKS_OK;
}

static ConstRes const_residues(const ckks_ctx* ctx, int level, int64_t m) {
  ConstRes r;
  for (int l = 0; l < level; ++l) {
    const u64 q = ctx->primes[l];
    const u64 mag = (u64)(m < 0 ? -(m + 1) : m) % q;  // |m| - [m < 0] avoids overflow at INT64_MIN
    u64 v = m < 0 ? (q - (mag + 1) % q) % q : mag;
    r.w[l] = v;
    r.ws[l] = h_shoup(v, q);
  }
  return r;
}

extern "C" int ckks_ct_add(const ckks_ctx* ctx, uint64_t* out, const uint64_t* a, const uint64_t* b, int n_ct,
                           int level, int subtract, void* stream) {
  const char* fn = "ckks_ct_add";
  if (int rc = check_ct(ctx, n_ct, level, fn)) return rc;
  const long long total = (long long)n_ct * 2 * level << ctx->log_n;
  if (total == 0) return CKKS_OK;
  CKKS_REQUIRE(out && a && b, "%s: NULL pointer argument", fn);
  k_ct_addsub<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(a), reinterpret_cast<const u64*>(b), total,
      ctx->log_n, level, subtract ? 1 : 0, ctx->d_pi);
  return ckks_check_launch(fn);
}

extern "C" int ckks_ct_mul_const(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_ct, int level,
                                 int64_t m, void* stream) {
  const char* fn = "ckks_ct_mul_const";
  if (int rc = check_ct(ctx, n_ct, level, fn)) return rc;
  const long long total = (long long)n_ct * 2 * level << ctx->log_n;
  if (total == 0) return CKKS_OK;
  CKKS_REQUIRE(out && in, "%s: NULL pointer argument", fn);
  k_ct_mul_const<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), total, ctx->log_n, level,
      const_residues(ctx, level, m), ctx->d_pi);
  return ckks_check_launch(fn);
}

extern "C" int ckks_ct_add_const(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_ct, int level,
                                 const uint64_t* c_res, void* stream) {
  const char* fn = "ckks_ct_add_const";
  if (int rc = check_ct(ctx, n_ct, level, fn)) return rc;
  CKKS_REQUIRE(c_res != nullptr, "%s: c_res is NULL", fn);
  ConstRes C;
  for (int l = 0; l < level; ++l) {
    CKKS_REQUIRE(c_res[l] < ctx->primes[l], "%s: c_res[%d] is not a residue mod q_%d", fn, l, l);
    C.w[l] = c_res[l];
    C.ws[l] = 0;
  }
  const long long total = (long long)n_ct * 2 * level << ctx->log_n;
  if (total == 0) return CKKS_OK;
  CKKS_REQUIRE(out && in, "%s: NULL pointer argument", fn);
  k_ct_add_const<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), total, ctx->log_n, level, C,
      ctx->d_pi);
  return ckks_check_launch(fn);
}
