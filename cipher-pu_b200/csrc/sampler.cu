// sampler.cu - seeded counter-based sampling for keys and encryption.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): a 4x32-bit counter is mixed with a 2x32-bit key
// through ten rounds of two 32x32->64 multiplies and xors, the key bumped by
// the Weyl constants between rounds.  Output word i of element idx depends
// only on (seed, stream, idx), so any launch shape reproduces the same values.
//  * uniform residues mod q: floor(u64 * q / 2^64) (bias < q / 2^64)
//  * ternary: floor(u64 * 3 / 2^64) - 1 (each of -1, 0, 1 with probability
//    1/3 up to 2^-64)
//  * discrete Gaussian, sigma <= 16, tail cut at 12 sigma: inverse CDF by
//    binary search in a 64-bit fixed-point table built on the host.
#include <cmath>
#include <vector>

#include "dispatch.cuh"

struct Philox {
  uint32_t c[4];
};

__device__ __forceinline__ void philox_round(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
  const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
  const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
  c[0] = n0;
  c[1] = n1;
  c[2] = n2;
  c[3] = n3;
}

__device__ __forceinline__ void philox4x32_10(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k0, k1);
    k0 += W0;
    k1 += W1;
  }
}

// two 64-bit words for element idx of stream `stream`
__device__ __forceinline__ void rand2x64(u64 seed, u64 stream, u64 idx, u64& a, u64& b) {
  uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  a = ((u64)c[1] << 32) | c[0];
  b = ((u64)c[3] << 32) | c[2];
}

__global__ void k_uniform(u64* __restrict__ out, long long total, int log_n, int n_limbs,
                          int prime_begin, const PrimeInfo* __restrict__ pi, u64 seed, u64 stream) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int limb = (int)((idx >> log_n) % n_limbs);
  const u64 q = pi[prime_begin + limb].q;
  u64 a, b;
  rand2x64(seed, stream, (u64)idx, a, b);
  out[idx] = __umul64hi(a, q);
}

__global__ void k_ternary(long long* __restrict__ out, long long n, u64 seed, u64 stream) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  u64 a, b;
  rand2x64(seed, stream, (u64)idx, a, b);
  // map the top 62 bits uniformly onto {0, 1, 2} by a 3 * 2^62 / 2^64 scaling
  const u64 t = __umul64hi(a, 3ull);
  out[idx] = (long long)t - 1;
}

__global__ void k_dgauss(long long* __restrict__ out, long long n, const u64* __restrict__ cdf,
                         int tail, u64 seed, u64 stream) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  u64 a, b;
  rand2x64(seed, stream, (u64)idx, a, b);
  // cdf[k] = P(X <= k - tail) in 2^64 fixed point, k = 0 .. 2 tail
  int lo = 0, hi = 2 * tail;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a <= cdf[mid]) hi = mid;
    else lo = mid + 1;
  }
  out[idx] = (long long)lo - tail;
}

extern "C" int ckks_sample_uniform(const ckks_ctx* ctx, uint64_t* out, int n_polys, int prime_begin,
                                   int n_limbs, uint64_t seed, uint64_t stream_id, void* stream) {
  CKKS_REQUIRE(ctx != nullptr, "ckks_sample_uniform: ctx is NULL");
  CKKS_REQUIRE(n_limbs >= 1 && prime_begin >= 0 && prime_begin + n_limbs <= ctx->n_primes,
               "ckks_sample_uniform: limb range outside the context");
  const long long total = ((long long)n_polys * n_limbs) << ctx->log_n;
  if (total <= 0) return CKKS_OK;
  k_uniform<<<grid1d((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), total, ctx->log_n, n_limbs, prime_begin, ctx->d_pi, seed,
      stream_id);
  return ckks_check_launch("ckks_sample_uniform");
}

extern "C" int ckks_sample_ternary(int64_t* out, int64_t n, uint64_t seed, uint64_t stream_id,
                                   void* stream) {
  CKKS_REQUIRE(n >= 0, "ckks_sample_ternary: n < 0");
  if (n == 0) return CKKS_OK;
  k_ternary<<<grid1d((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<long long*>(out), n, seed, stream_id);
  return ckks_check_launch("ckks_sample_ternary");
}

namespace {
struct CdfTable {
  double sigma = -1.0;
  int tail = 0;
  u64* d = nullptr;
  int device = -1;
};
thread_local CdfTable g_cdf;
}  // namespace

extern "C" int ckks_sample_dgauss(int64_t* out, int64_t n, double sigma, uint64_t seed,
                                  uint64_t stream_id, void* stream) {
  CKKS_REQUIRE(n >= 0, "ckks_sample_dgauss: n < 0");
  CKKS_REQUIRE(sigma > 0.0 && sigma <= 16.0, "ckks_sample_dgauss: sigma outside (0, 16]");
  if (n == 0) return CKKS_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_cdf.sigma != sigma || g_cdf.device != dev) {
    const int tail = (int)std::ceil(12.0 * sigma);
    std::vector<long double> w(2 * tail + 1);
    long double z = 0;
    for (int k = -tail; k <= tail; ++k) {
      w[k + tail] = std::exp(-(long double)k * k / (2.0L * sigma * sigma));
      z += w[k + tail];
    }
    std::vector<u64> cdf(2 * tail + 1);
    long double acc = 0;
    for (int i = 0; i <= 2 * tail; ++i) {
      acc += w[i] / z;
      const long double v = acc * 18446744073709551616.0L;
      cdf[i] = v >= 18446744073709551615.0L ? ~0ull : (u64)v;
    }
    cdf[2 * tail] = ~0ull;
    if (g_cdf.d && g_cdf.device == dev) cudaFree(g_cdf.d);
    u64* d = nullptr;
    cudaError_t e = cudaMalloc(&d, cdf.size() * sizeof(u64));
    if (e == cudaSuccess) e = cudaMemcpy(d, cdf.data(), cdf.size() * sizeof(u64), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_sample_dgauss: %s", cudaGetErrorString(e));
    g_cdf.d = d;
    g_cdf.sigma = sigma;
    g_cdf.tail = tail;
    g_cdf.device = dev;
  }
  k_dgauss<<<grid1d((n + 255) / 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<long long*>(out), n, g_cdf.d, g_cdf.tail, seed, stream_id);
  return ckks_check_launch("ckks_sample_dgauss");
}
