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
// Tiling (k_linear below): a modular GEMM tile of 32 outputs x 128 positions
// per CTA, 4 x 4 accumulator pairs per thread, input tiles double-buffered in
// shared memory by cp.async.  Skipped 4x4 weight blocks cost nothing, and an
// input column block that no row block of the CTA keeps is never loaded, so
// both the multiplies and the input traffic scale with the kept fraction.
#include "dispatch.cuh"
#include "profile.hpp"

constexpr int LIN_ROWB = 8;                  // 4-row blocks per CTA (one per warp)
constexpr int LIN_OT = 4 * LIN_ROWB;         // outputs per CTA
constexpr int LIN_PT = 128;                  // positions per CTA (4 per lane)
constexpr int LIN_THREADS = 32 * LIN_ROWB;
constexpr int LIN_CB = 8;                    // column blocks (4 inputs each) per pipeline chunk
constexpr int LIN_MAX_IN = 2048;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
               "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND)); }

// acc += a * b with a 32 x 32 -> 64-bit signed multiply-add
__device__ __forceinline__ void mad_wide(long long& acc, int a, int b) {
  asm("mad.wide.s32 %0, %1, %2, %0;" : "+l"(acc) : "r"(a), "r"(b));
}

struct LinSmem {
  u64 x[2][LIN_CB * 4][LIN_PT];   // input tiles: [buffer][input slot][position]
  int w[2][LIN_CB * 4][LIN_OT];   // weight tiles: [buffer][input slot][output]
  unsigned char keep[2][LIN_CB][LIN_ROWB];
  int cbl[LIN_MAX_IN / 4];        // column blocks some row block of the CTA keeps
  int ncb;
};

// One CTA = 32 outputs x 128 positions; warp r owns outputs o0 + 4r .. + 3
// (one 4-row block, so the block-keep test is warp-uniform), lane l owns
// positions p0 + 2l, +1 and p0 + 64 + 2l, +1 (16-byte shared loads that are
// contiguous across the warp: no bank conflicts).  The input column blocks that none of the CTA's
// row blocks keeps are skipped entirely (neither loaded nor multiplied); the
// others stream through a two-stage cp.async pipeline of LIN_CB blocks.
__global__ void __launch_bounds__(LIN_THREADS, 2)
    k_linear(u64* __restrict__ out, const u64* __restrict__ in, const int* __restrict__ w,
             const long long* __restrict__ bias, const unsigned char* __restrict__ keep, int n_out,
             int n_in, int level, int log_n, const PrimeInfo* __restrict__ pi) {
  extern __shared__ __align__(16) unsigned char lin_raw[];
  LinSmem& S = *reinterpret_cast<LinSmem*>(lin_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int o0 = blockIdx.x * LIN_OT;  // output tiles vary fastest: they share the input tile in L2
  const long long npos = (2ll * level) << log_n;
  const long long p0 = (long long)blockIdx.y * LIN_PT;
  const int nb_in = (n_in + 3) / 4;
  const int rb0 = o0 / 4;
  const int nrb = (n_out + 3) / 4;
  auto kept = [&](int rb, int cb) -> bool {
    if (rb >= nrb) return false;
    return keep ? keep[(size_t)rb * nb_in + cb] != 0 : true;
  };
  // compact list of the column blocks this CTA needs (warp 0, ballot scan)
  if (warp == 0) {
    int base = 0;
    for (int c0 = 0; c0 < nb_in; c0 += 32) {
      const int cb = c0 + lane;
      bool need = false;
      if (cb < nb_in)
        for (int r = 0; r < LIN_ROWB; ++r) need |= kept(rb0 + r, cb);
      const unsigned m = __ballot_sync(0xffffffffu, need);
      if (need) S.cbl[base + __popc(m & ((1u << lane) - 1))] = cb;
      base += __popc(m);
    }
    if (lane == 0) S.ncb = base;
  }
  __syncthreads();
  const int ncb = S.ncb;
  const int nchunk = (ncb + LIN_CB - 1) / LIN_CB;

  // stage chunk c into buffer b: inputs by cp.async, weights and keep bits by plain loads
  auto stage_x = [&](int c, int b) {
#pragma unroll
    for (int u = 0; u < (LIN_CB * 4 * LIN_PT * 8) / (16 * LIN_THREADS); ++u) {
      const int idx = tid + LIN_THREADS * u;           // 16-byte piece
      const int row = idx / (LIN_PT / 2), col = idx % (LIN_PT / 2);
      const int j = row >> 2, t = row & 3;
      const int ci = c * LIN_CB + j;
      const int f = ci < ncb ? 4 * S.cbl[ci] + t : n_in;
      const long long p = p0 + 2 * col;
      const bool valid = f < n_in && p < npos;
      const u64* src = valid ? in + (size_t)f * npos + p : in;
      cp_async16(&S.x[b][row][2 * col], src, valid);
    }
  };
  auto load_w = [&](int c, int (&wr)[(LIN_CB * 4 * LIN_OT) / LIN_THREADS]) {
#pragma unroll
    for (int u = 0; u < (LIN_CB * 4 * LIN_OT) / LIN_THREADS; ++u) {
      const int idx = tid + LIN_THREADS * u;
      const int row = idx / LIN_OT, o = idx % LIN_OT;
      const int ci = c * LIN_CB + (row >> 2);
      const int f = ci < ncb ? 4 * S.cbl[ci] + (row & 3) : n_in;
      wr[u] = (f < n_in && o0 + o < n_out) ? __ldg(w + (size_t)(o0 + o) * n_in + f) : 0;
    }
  };
  auto store_w = [&](int c, int b, const int (&wr)[(LIN_CB * 4 * LIN_OT) / LIN_THREADS]) {
#pragma unroll
    for (int u = 0; u < (LIN_CB * 4 * LIN_OT) / LIN_THREADS; ++u) {
      const int idx = tid + LIN_THREADS * u;
      S.w[b][idx / LIN_OT][idx % LIN_OT] = wr[u];
    }
    if (tid < LIN_CB * LIN_ROWB) {
      const int j = tid / LIN_ROWB, r = tid % LIN_ROWB;
      const int ci = c * LIN_CB + j;
      S.keep[b][j][r] = ci < ncb ? (kept(rb0 + r, S.cbl[ci]) ? 1 : 0) : 0;
    }
  };

  long long al[4][4], ah[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int i = 0; i < 4; ++i) al[r][i] = ah[r][i] = 0;
  const u64 mask23 = (1ull << 23) - 1;
  int wr[(LIN_CB * 4 * LIN_OT) / LIN_THREADS];
  if (nchunk > 0) {
    stage_x(0, 0);
    cp_async_commit();
    load_w(0, wr);
    store_w(0, 0, wr);
  }
#pragma unroll 1
  for (int c = 0; c < nchunk; ++c) {
    const int b = c & 1;
    const bool more = c + 1 < nchunk;
    if (more) {
      stage_x(c + 1, b ^ 1);
      cp_async_commit();
      load_w(c + 1, wr);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll 1
    for (int j = 0; j < LIN_CB; ++j) {
      if (!S.keep[b][j][warp]) continue;  // warp-uniform
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int row = 4 * j + t;
        const int4 wv = *reinterpret_cast<const int4*>(&S.w[b][row][4 * warp]);
        const ulonglong2 xa = *reinterpret_cast<const ulonglong2*>(&S.x[b][row][2 * lane]);
        const ulonglong2 xb = *reinterpret_cast<const ulonglong2*>(&S.x[b][row][LIN_PT / 2 + 2 * lane]);
        const u64 xv[4] = {xa.x, xa.y, xb.x, xb.y};
        const int wvv[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          // 32 x 32 -> 64-bit multiply-adds (one IMAD.WIDE each): both halves
          // of the residue fit in 24 bits, the weights in 24 bits
          const int xl = (int)(xv[i] & mask23), xh = (int)(xv[i] >> 23);
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            mad_wide(al[r][i], wvv[r], xl);
            mad_wide(ah[r][i], wvv[r], xh);
          }
        }
      }
    }
    if (more) store_w(c + 1, b ^ 1, wr);
    __syncthreads();
  }
  // epilogue: reduce, add the bias on component 0, store the two word pairs
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const long long pl = p0 + h * (LIN_PT / 2) + 2 * lane;
    if (pl >= npos) continue;
    const int limb = (int)((pl >> log_n) % level);
    const int comp = (int)(pl / ((long long)level << log_n));
    const PrimeInfo P = pi[limb];
    const long long qs = (long long)P.q;
    const u64 two23 = (1ull << 23) % P.q;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int o = o0 + 4 * warp + r;
      if (o >= n_out) break;
      long long bq = 0;
      if (bias && comp == 0) {
        bq = bias[o] % qs;
        if (bq < 0) bq += qs;
      }
      u64 v[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        long long rl = al[r][2 * h + i] % qs;
        if (rl < 0) rl += qs;
        long long rh = ah[r][2 * h + i] % qs;
        if (rh < 0) rh += qs;
        v[i] = addmod(addmod(mulmod((u64)rh, two23, P), (u64)rl, P.q), (u64)bq, P.q);
      }
      *reinterpret_cast<ulonglong2*>(out + (size_t)o * npos + pl) = make_ulonglong2(v[0], v[1]);
    }
  }
}

extern "C" int ckks_linear_plain_weights(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in,
                                         const int32_t* w, const int64_t* bias,
                                         const uint8_t* block_keep, int n_out, int n_in, int level,
                                         void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks linear layer (integer pipe)");
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
  dim3 grid((unsigned)((n_out + LIN_OT - 1) / LIN_OT), (unsigned)((npos + LIN_PT - 1) / LIN_PT));
  CKKS_REQUIRE(grid.y <= 65535, "%s: too many positions (2 level N / %d > 65535)", fn, LIN_PT);
  const int smem = (int)sizeof(LinSmem);
  if (cudaError_t e = ensure_smem(k_linear, smem))
    return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  k_linear<<<grid, LIN_THREADS, smem, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), w,
      reinterpret_cast<const long long*>(bias), block_keep, n_out, n_in, level, ctx->log_n, ctx->d_pi);
  return ckks_check_launch(fn);
}
