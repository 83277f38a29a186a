// linear.cu - encrypted linear layer with plaintext integer weights and
// 4x4 block sparsity (the FC layer of the encrypted MLP / CNN).
//
//   out[o] = sum_f w[o][f] * in[f]  (+ bias[o] on component 0)   mod q_i
//
// Ciphertexts are [count][2][level][N] in the evaluation domain; the weight of
// a ciphertext-times-scalar product is the same in every limb and every slot,
// so the layer is a modular GEMM over the 2 * level * N coefficient positions.
// Exactness: each residue x < 2^47 is split x = xh 2^23 + xl, products with
// |w| < 2^24 are accumulated in signed 64-bit (|sum| < 2^57 for <= 1024
// inputs; |sum| < 2^59 for 2048), reduced once per output element.
//
// Tiling: one CTA = 16 outputs (four 4-row blocks) x 256 positions, one
// position per thread; the weight tile and the block-keep mask live in
// shared memory.  A 4-input column block is loaded only when one of the four
// row blocks keeps it, and each kept 4x4 block costs 16 x 2 IMAD.WIDE per
// position, so the work scales with the kept fraction.
#include "dispatch.cuh"

constexpr int LIN_OT = 16;     // outputs per CTA
constexpr int LIN_THREADS = 256;
constexpr int LIN_MAX_IN = 2048;

__global__ void __launch_bounds__(LIN_THREADS)
    k_linear(u64* __restrict__ out, const u64* __restrict__ in, const int* __restrict__ w,
             const long long* __restrict__ bias, const unsigned char* __restrict__ keep, int n_out,
             int n_in, int level, int log_n, const PrimeInfo* __restrict__ pi) {
  extern __shared__ int lin_sm[];
  const int o0 = blockIdx.y * LIN_OT;
  const int nb_in = (n_in + 3) / 4;
  const int ldw = 4 * nb_in;  // padded row length of the weight tile
  int* ws = lin_sm;                                                   // [LIN_OT][ldw]
  unsigned char* ks = reinterpret_cast<unsigned char*>(lin_sm + LIN_OT * ldw);  // [4][nb_in]
  for (int t = threadIdx.x; t < LIN_OT * ldw; t += blockDim.x) {
    const int r = t / ldw, f = t % ldw;
    ws[t] = (o0 + r < n_out && f < n_in) ? w[(size_t)(o0 + r) * n_in + f] : 0;
  }
  for (int t = threadIdx.x; t < 4 * nb_in; t += blockDim.x) {
    const int rb = t / nb_in, cb = t % nb_in;
    const int orb = o0 / 4 + rb;
    unsigned char k = 0;
    if (o0 + 4 * rb < n_out) k = keep ? keep[(size_t)orb * nb_in + cb] : 1;
    ks[t] = k;
  }
  __syncthreads();
  const long long npos = (2ll * level) << log_n;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npos) return;
  const int limb = (int)((p >> log_n) % level);
  const int comp = (int)(p / ((long long)level << log_n));
  long long al[LIN_OT], ah[LIN_OT];
#pragma unroll
  for (int o = 0; o < LIN_OT; ++o) al[o] = ah[o] = 0;
  const u64 mask23 = (1ull << 23) - 1;
#pragma unroll 1
  for (int cb = 0; cb < nb_in; ++cb) {
    const unsigned char k0 = ks[cb], k1 = ks[nb_in + cb], k2 = ks[2 * nb_in + cb],
                        k3 = ks[3 * nb_in + cb];
    if (!(k0 | k1 | k2 | k3)) continue;
    long long xl[4], xh[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int f = 4 * cb + t;
      const u64 x = f < n_in ? __ldg(in + (size_t)f * npos + p) : 0ull;
      xl[t] = (long long)(x & mask23);
      xh[t] = (long long)(x >> 23);
    }
#pragma unroll
    for (int rb = 0; rb < 4; ++rb) {
      const unsigned char kk = rb == 0 ? k0 : rb == 1 ? k1 : rb == 2 ? k2 : k3;
      if (!kk) continue;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int o = 4 * rb + r;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const long long wv = ws[o * ldw + 4 * cb + t];
          al[o] += wv * xl[t];
          ah[o] += wv * xh[t];
        }
      }
    }
  }
  const PrimeInfo P = pi[limb];
  const long long qs = (long long)P.q;
  const u64 two23 = (1ull << 23) % P.q;
#pragma unroll
  for (int o = 0; o < LIN_OT; ++o) {
    if (o0 + o >= n_out) break;
    long long rl = al[o] % qs;
    if (rl < 0) rl += qs;
    long long rh = ah[o] % qs;
    if (rh < 0) rh += qs;
    u64 v = addmod(mulmod((u64)rh, two23, P), (u64)rl, P.q);
    if (bias && comp == 0) {
      long long b = bias[o0 + o] % qs;
      if (b < 0) b += qs;
      v = addmod(v, (u64)b, P.q);
    }
    out[(size_t)(o0 + o) * npos + p] = v;
  }
}

extern "C" int ckks_linear_plain_weights(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in,
                                         const int32_t* w, const int64_t* bias,
                                         const uint8_t* block_keep, int n_out, int n_in, int level,
                                         void* stream) {
  const char* fn = "ckks_linear_plain_weights";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_in >= 1 && n_in <= LIN_MAX_IN, "%s: n_in=%d outside [1, %d]", fn, n_in, LIN_MAX_IN);
  CKKS_REQUIRE(n_out >= 1, "%s: n_out=%d < 1", fn, n_out);
  CKKS_REQUIRE(level >= 1 && level <= ctx->n_primes, "%s: level=%d outside [1, %d]", fn, level,
               ctx->n_primes);
  for (int i = 0; i < level; ++i)
    CKKS_REQUIRE(ctx->primes[i] < (1ull << 47), "%s: primes must be below 2^47", fn);
  CKKS_REQUIRE(out && in && w, "%s: NULL pointer argument", fn);
  CKKS_REQUIRE((const void*)out != (const void*)in, "%s: out must differ from in", fn);
  const long long npos = (2ll * level) << ctx->log_n;
  dim3 grid((unsigned)((npos + LIN_THREADS - 1) / LIN_THREADS), (unsigned)((n_out + LIN_OT - 1) / LIN_OT));
  CKKS_REQUIRE(grid.y <= 65535, "%s: n_out too large", fn);
  const int nb_in = (n_in + 3) / 4;
  const int smem = LIN_OT * 4 * nb_in * (int)sizeof(int) + 4 * nb_in;
  if (cudaError_t e = ensure_smem(k_linear, smem))
    return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  k_linear<<<grid, LIN_THREADS, smem, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), w,
      reinterpret_cast<const long long*>(bias), block_keep, n_out, n_in, level, ctx->log_n, ctx->d_pi);
  return ckks_check_launch(fn);
}
