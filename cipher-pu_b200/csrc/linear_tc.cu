// linear_tc.cu - the encrypted linear layer on the 5th-generation tensor cores
// (tcgen05.mma, kind::i8, accumulators in TMEM).
//
//   out[o][p] = sum_f w[o][f] x[f][p]  (+ bias[o] on component 0)   mod q_limb(p)
//
// x are ciphertext residues (< 2^48) at the 2 level N positions of each input
// ciphertext, w plaintext integer weights.  Exact integer arithmetic through
// byte limbs: x = sum_a x_a 256^a with unsigned bytes x_a (a < 6), w = sum_b
// w_b 256^b with balanced signed bytes w_b in [-128, 127] (b < 3, so
// |w| <= 127 (1 + 256 + 256^2) = 8355711 < 2^23).  The 18 limb products
// w_b x x_a are int8 x uint8 GEMMs with exact int32 accumulation; the ones with
// the same a + b = c share one accumulator D_c (8 of them, |D_c| < 3 * 2048 *
// 128 * 255 < 2^28 for n_in <= 2048), and the epilogue forms
// sum_c D_c [256^c]_q (+ bias) exactly in FP64 and reduces it mod q.
//
// Tiling (16 loader warps + 1 MMA-issuing warp): one CTA per 128 outputs (the MMA's M) x 64 positions (its N; the
// epilogue finds each group of 8 positions' limb, so N may be below 64);
// features in chunks of 128 (bytes per operand row), two
// shared-memory stages.  For each chunk every thread loads uint64 residues
// (4 features x 1 position each, coalesced along positions) and writes their
// six byte planes straight into the operand images; the weights arrive as a
// pre-packed image of the same layout (ckks_linear_tc_pack, host side, once
// per weight matrix and block mask).  The issuer warp's first thread then
// issues the chunk's 3 x 6 x 4 MMAs (M 128, N 64, K 32) and commits them to
// the stage's mbarrier while the loader warps go on to fill the other stage; a stage is refilled only after its previous MMAs' commit
// (bounded wait).  TMEM: 8 accumulators x 64 columns = all 512 columns, one
// CTA per SM (its 192 KB of shared memory guarantees that).
//
// Operand images, K-major without swizzle (the UMMA canonical
// "interleave" layout): core matrices of 8 rows x 16 bytes (128 B,
// contiguous), the two 16-byte halves of a 32-byte K step LBO = 128 B apart,
// 8-row groups SBO = 1024 B apart (a row holds the chunk's 128 K bytes).
#include <cstring>

#include "dispatch.cuh"
#include "tmem.cuh"
#include "umma.cuh"
#include "profile.hpp"

namespace {

constexpr int TC_M = 128;                     // outputs per tile (MMA M)
constexpr int TC_N = 64;                      // positions per tile (MMA N)
constexpr int TC_KC = 128;                    // features per chunk
constexpr int TC_WL = 3;                      // signed weight byte limbs
constexpr int TC_XL = 6;                      // unsigned residue byte limbs
constexpr int TC_ACC = TC_WL + TC_XL - 1;     // accumulators D_c, c = a + b
constexpr int TC_LOADERS = 512;               // threads that load / split operands and run the epilogue
constexpr int TC_THREADS = TC_LOADERS + 32;   // plus one warp that issues the MMAs
constexpr int TC_ISSUER = TC_LOADERS;         // its first thread
constexpr int TC_A_IMG = TC_M * TC_KC;        // 16 KB: one weight limb of one chunk
constexpr int TC_B_IMG = TC_N * TC_KC;        // 8 KB: one residue limb of one chunk
constexpr int TC_STAGE = TC_WL * TC_A_IMG + TC_XL * TC_B_IMG;  // 96 KB
constexpr int TC_SMEM = 2 * TC_STAGE;         // 192 KB
constexpr int TC_MAX_IN = 2048;
constexpr long long TC_W_MAX = 127ll * (1 + 256 + 65536);   // largest |w| of 3 balanced limbs
constexpr int TC_OUT_STRIDE = TC_N + 1;       // staging row stride (u64), breaks bank aliasing
static_assert(TC_ACC * TC_N <= 512, "accumulators exceed the TMEM columns");
static_assert(TC_M * TC_OUT_STRIDE * 8 <= TC_SMEM, "output staging must fit the stages");

// byte offset of (row, k) in an operand image
__host__ __device__ constexpr int img_off(int row, int k) {
  return (row >> 3) * (8 * TC_KC) + (k >> 4) * 128 + (row & 7) * 16 + (k & 15);
}

__device__ unsigned int g_tc_wait_expiries;

// instruction descriptor: D s32, A s8 (weights), B u8 (residue bytes), both
// K-major, N = 64, M = 128, dense
constexpr uint32_t kTcIdesc = (2u << 4) | (1u << 7) | (0u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate)
      : "memory");
}
}  // namespace

__global__ void __launch_bounds__(TC_THREADS, 1)
    k_linear_tc(u64* __restrict__ out, const u64* __restrict__ in, const unsigned char* __restrict__ wpk,
                const long long* __restrict__ bias, int n_out, int n_in, int level, int log_n,
                const PrimeInfo* __restrict__ pi, long long wait_limit) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(8) unsigned long long bars[2];
  __shared__ __align__(8) unsigned long long wbars[2];  // weight image of a stage landed
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int mt = blockIdx.y;
  const long long npos = (2ll * level) << log_n;
  const long long p0 = (long long)blockIdx.x * TC_N;
  const int nchunk = (n_in + TC_KC - 1) / TC_KC;
  const uint32_t bar[2] = {s_u32(&bars[0]), s_u32(&bars[1])};
  const uint32_t wbar[2] = {s_u32(&wbars[0]), s_u32(&wbars[1])};

  if (warp == 0) tmem_alloc_warp(&tmem_slot, 512);
  if (tid == 32) {
    tc_mbar_init(bar[0]);
    tc_mbar_init(bar[1]);
    tc_mbar_init(wbar[0]);
    tc_mbar_init(wbar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tbase = tmem_slot;

  // commits issued / waited for per stage (the k-th completion has parity k & 1)
  int n_commit[2] = {0, 0}, n_waited[2] = {0, 0};
  // thread 0: a weight copy issued and not yet seen landed (stage, parity), or -1
  int w_pending = -1;
  bool ok = true;
#pragma unroll 1
  for (int kc = 0; kc < nchunk; ++kc) {
    const int s = kc & 1;
    unsigned char* A = smem + s * TC_STAGE;
    unsigned char* Bm = A + TC_WL * TC_A_IMG;
    // the MMAs of chunk kc - 2 may still read this stage: every loader thread
    // polls its commit (bounded) and proceeds on its own; the issuer warp,
    // meanwhile still issuing chunk kc - 1, is not waited for here
    const bool need_wait = n_waited[s] < n_commit[s];
    bool expired = false;
    if (tid < TC_LOADERS && need_wait) expired = !tc_mbar_wait(bar[s], n_waited[s] & 1, wait_limit);
    const uint32_t wpar = (uint32_t)(kc >> 1) & 1u;  // this stage's use number kc / 2, mod 2
    if (tid < TC_LOADERS && !expired) {
      // weight limbs: the packed image of (tile mt, chunk kc), already in the
      // UMMA layout, as one bulk asynchronous copy (the stage is free: this
      // thread has just seen its previous MMAs complete)
      if (tid == 0) {
        tc_bulk_load(s_u32(A), wpk + ((size_t)mt * nchunk + kc) * TC_WL * TC_A_IMG, TC_WL * TC_A_IMG, wbar[s]);
        w_pending = s * 2 + (int)wpar;
      }
      // residue limbs: 64 tasks (8 position x 8 feature groups), 4 per warp;
      // lane = 8 fq + pl takes position pb + pl and features fb + 4 fq .. + 3,
      // so a warp's 4-byte image stores hit 32 distinct banks.  Every load of
      // the chunk is issued before the first is used (16 per thread in flight).
      constexpr int TPW = 64 / (TC_LOADERS / 32);  // tasks per loader warp
      u64 xv[TPW][4];
  #pragma unroll
      for (int it = 0; it < TPW; ++it) {
        const int task = warp * TPW + it;
        const int p = (task & 7) * 8 + (lane & 7);
        const int f = kc * TC_KC + (task >> 3) * 16 + 4 * (lane >> 3);
  #pragma unroll
        for (int t = 0; t < 4; ++t)
          xv[it][t] = (f + t < n_in) ? ld_stream(in + (size_t)(f + t) * npos + p0 + p) : 0ull;
      }
  #pragma unroll
      for (int it = 0; it < TPW; ++it) {
        const int task = warp * TPW + it;
        const int p = (task & 7) * 8 + (lane & 7);
        const int fl = (task >> 3) * 16 + 4 * (lane >> 3);
        // byte transpose: plane a, byte t = byte a of residue t (feature fl + t)
        uint32_t pl[TC_XL];
        byte_planes(xv[it], pl);
        const int off = img_off(p, fl);
  #pragma unroll
        for (int a = 0; a < TC_XL; ++a) *reinterpret_cast<uint32_t*>(Bm + a * TC_B_IMG + off) = pl[a];
      }
    }
    // the weight image has landed (bounded wait)
    if (tid == 0 && w_pending >= 0) {
      if (tc_mbar_wait(wbar[s], wpar, wait_limit)) w_pending = -1;
      else expired = true;
    }
    // make the generic-proxy stores visible to the tensor cores, then issue
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (__syncthreads_or(expired)) {
      ok = false;
      break;
    }
    if (need_wait) ++n_waited[s];
    if (tid == TC_ISSUER) {
      tmem_fence_after_sync();
      // observe the weight copy's completion here too (already complete:
      // thread 0 saw it before the barrier), ordering it before the MMAs
      tc_mbar_wait(wbar[s], wpar, wait_limit);
      // descriptors of the stage's first operand rows; later ones differ only
      // in the start-address field (byte offset / 16, no carry below 256 KB)
      const uint64_t da = umma_desc(s_u32(A), 128, 8 * TC_KC);
      const uint64_t db = umma_desc(s_u32(Bm), 128, 8 * TC_KC);
#pragma unroll
      for (int b = 0; b < TC_WL; ++b)
#pragma unroll
        for (int a = 0; a < TC_XL; ++a) {
          const int c = a + b;
          const bool first = b == (c > TC_XL - 1 ? c - (TC_XL - 1) : 0);  // first pair of D_c
#pragma unroll
          for (int ks = 0; ks < TC_KC / 32; ++ks)
            tc_mma(tbase + (uint32_t)(c * TC_N), da + (uint64_t)((b * TC_A_IMG + ks * 256) >> 4),
                   db + (uint64_t)((a * TC_B_IMG + ks * 256) >> 4),
                   (kc == 0 && first && ks == 0) ? 0u : 1u);
        }
      tc_commit(bar[s]);
    }
    ++n_commit[s];
  }
  // the last chunk's commit covers every MMA issued before it; on an expired
  // wait, drain every outstanding commit instead (bounded) so nothing is in
  // flight when the CTA leaves
  // (at most one commit per stage is ever outstanding: a stage is refilled
  // only after its previous commit has been waited for)
  if (ok && nchunk > 0) {
    const int s = (nchunk - 1) & 1;
    bool w = true;
    if (tid == TC_ISSUER) w = tc_mbar_wait(bar[s], n_waited[s] & 1, wait_limit);
    if (__syncthreads_or(!w)) ok = false;
    else ++n_waited[s];
  }
  if (!ok && tid == 0 && w_pending >= 0 && !tc_mbar_wait(wbar[w_pending >> 1], w_pending & 1, kTcDrainCycles))
    atomicAdd(&g_tc_wait_expiries, 1u);  // a weight copy still in flight after the drain limit
  if (!ok && tid == TC_ISSUER) {
    atomicAdd(&g_tc_wait_expiries, 1u);
    for (int st = 0; st < 2; ++st)
      if (n_waited[st] < n_commit[st] && !tc_mbar_wait(bar[st], n_waited[st] & 1, kTcDrainCycles))
        atomicAdd(&g_tc_wait_expiries, 1u);  // still in flight after the drain limit
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();

  if (ok && tid < TC_LOADERS) {
    // epilogue: thread (warp w, lane l) owns output row r = 32 (w mod 4) + l;
    // the warps of one lane quarter take the groups of 8 positions in turn
    const int r = (warp & 3) * 32 + lane;
    const int o = mt * TC_M + r;
    const long long bias_o = (bias != nullptr && o < n_out) ? bias[o] : 0;
    u64* stage = reinterpret_cast<u64*>(smem);
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
#pragma unroll 1
    for (int g = warp >> 2; g < TC_N / 8; g += TC_LOADERS / 128) {
      // a group of 8 positions lies in one limb and one component (N >= 8);
      // a tile may span several when N < 64
      const long long pg = p0 + 8 * g;
      const int limb = (int)((pg >> log_n) % level);
      const int comp = (int)(pg / ((long long)level << log_n));
      const PrimeInfo P = pi[limb];
      double bq = 0.0;
      if (comp == 0 && bias_o != 0) {
        long long b = bias_o % (long long)P.q;
        if (b < 0) b += (long long)P.q;
        bq = (double)b;
      }
      double acc[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = bq;
      u64 pw = 1ull % P.q;  // 256^c mod q
#pragma unroll
      for (int c = 0; c < TC_ACC; ++c) {
        const double wc = (double)pw, wq = __ddiv_rn(wc, P.qd);
        pw = (pw << 8) % P.q;
        int d[8];
        tmem_ld8_i32(tbase + lane_base + (uint32_t)(c * TC_N + 8 * g), d);
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = __dadd_rn(acc[j], fmulmod((double)d[j], wc, wq, P.qd));
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) stage[r * TC_OUT_STRIDE + 8 * g + j] = d2canon(acc[j], P.qd, P.qinv_d);
    }
    // the loader warps' named barrier (the issuer warp is not in this branch)
    asm volatile("bar.sync 1, %0;" ::"n"(TC_LOADERS) : "memory");
    // coalesced rows: warp w stores rows w, w + 16, ...; each lane 2 words
#pragma unroll 1
    for (int row = warp; row < TC_M; row += TC_LOADERS / 32) {
      const int orow = mt * TC_M + row;
      if (orow >= n_out) break;
      u64* dst = out + (size_t)orow * npos + p0;
      dst[lane] = stage[row * TC_OUT_STRIDE + lane];
      dst[lane + 32] = stage[row * TC_OUT_STRIDE + lane + 32];
    }
  }
  tmem_fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc_warp(tbase, 512);
}

// ------------------------------------------------------------------ host side
extern "C" size_t ckks_linear_tc_packed_bytes(int n_out, int n_in) {
  if (n_out < 1 || n_in < 1) return 0;
  const size_t mtiles = (size_t)(n_out + TC_M - 1) / TC_M;
  const size_t chunks = (size_t)(n_in + TC_KC - 1) / TC_KC;
  return mtiles * chunks * TC_WL * TC_A_IMG;
}

extern "C" int ckks_linear_tc_pack(void* packed, size_t packed_bytes, const int32_t* w,
                                   const uint8_t* block_keep, int n_out, int n_in) {
  const char* fn = "ckks_linear_tc_pack";
  CKKS_REQUIRE(n_out >= 1 && n_in >= 1 && n_in <= TC_MAX_IN, "%s: n_out=%d, n_in=%d (n_in <= %d)", fn,
               n_out, n_in, TC_MAX_IN);
  CKKS_REQUIRE(packed && w, "%s: NULL pointer argument", fn);
  const size_t need = ckks_linear_tc_packed_bytes(n_out, n_in);
  CKKS_REQUIRE(packed_bytes >= need, "%s: %zu bytes < %zu needed", fn, packed_bytes, need);
  const int nb_in = (n_in + 3) / 4;
  for (size_t i = 0; i < (size_t)n_out * n_in; ++i) {
    const long long v = w[i] < 0 ? -(long long)w[i] : (long long)w[i];
    CKKS_REQUIRE(v <= TC_W_MAX, "%s: |w[%zu]| = %lld exceeds %lld (three signed byte limbs)", fn, i, v,
                 TC_W_MAX);
  }
  unsigned char* img = static_cast<unsigned char*>(packed);
  memset(img, 0, need);
  const int chunks = (n_in + TC_KC - 1) / TC_KC;
  for (int o = 0; o < n_out; ++o)
    for (int f = 0; f < n_in; ++f) {
      if (block_keep && !block_keep[(size_t)(o / 4) * nb_in + f / 4]) continue;
      long long v = w[(size_t)o * n_in + f];
      const int mt = o / TC_M, row = o % TC_M, kc = f / TC_KC, k = f % TC_KC;
      unsigned char* tile = img + ((size_t)mt * chunks + kc) * TC_WL * TC_A_IMG;
      for (int b = 0; b < TC_WL; ++b) {
        long long d = v & 0xFF;        // balanced digit in [-128, 127]
        if (d > 127) d -= 256;
        v = (v - d) / 256;
        tile[b * TC_A_IMG + img_off(row, k)] = (unsigned char)(signed char)d;
      }
    }
  return CKKS_OK;
}

int ckks_linear_tc_status_take(unsigned int* n) {
  cudaError_t e = cudaMemcpyFromSymbol(n, g_tc_wait_expiries, sizeof(*n));
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  if (*n) {
    const unsigned int zero = 0;
    e = cudaMemcpyToSymbol(g_tc_wait_expiries, &zero, sizeof(zero));
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  }
  return CKKS_OK;
}

extern "C" int ckks_linear_plain_weights_tc(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in,
                                            const void* packed, const int64_t* bias, int n_out, int n_in,
                                            int level, void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks linear layer (tensor cores)");
  const char* fn = "ckks_linear_plain_weights_tc";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_in >= 1 && n_in <= TC_MAX_IN, "%s: n_in=%d outside [1, %d]", fn, n_in, TC_MAX_IN);
  CKKS_REQUIRE(n_out >= 1, "%s: n_out=%d < 1", fn, n_out);
  CKKS_REQUIRE(level >= 1 && level <= ctx->n_primes, "%s: level=%d outside [1, %d]", fn, level,
               ctx->n_primes);
  for (int i = 0; i < level; ++i)
    CKKS_REQUIRE(ctx->primes[i] < (1ull << 47), "%s: primes must be below 2^47", fn);
  CKKS_REQUIRE(ctx->log_n >= 5, "%s: N=2^%d below the 64-position tile (N >= 32)", fn, ctx->log_n);
  CKKS_REQUIRE(out && in && packed, "%s: NULL pointer argument", fn);
  CKKS_REQUIRE((const void*)out != (const void*)in, "%s: out must differ from in", fn);
  CKKS_REQUIRE((reinterpret_cast<uintptr_t>(packed) & 15) == 0, "%s: packed weights must be 16-byte aligned",
               fn);
  const long long npos = (2ll * level) << ctx->log_n;
  const dim3 grid((unsigned)(npos / TC_N), (unsigned)((n_out + TC_M - 1) / TC_M));
  CKKS_REQUIRE(grid.y <= 65535, "%s: too many output tiles", fn);
  if (int rc = require_smem(TC_SMEM + 64, ctx->log_n, fn)) return rc;
  if (cudaError_t e = ensure_smem(k_linear_tc, TC_SMEM))
    return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  k_linear_tc<<<grid, TC_THREADS, TC_SMEM, as_stream(stream)>>>(
      reinterpret_cast<u64*>(out), reinterpret_cast<const u64*>(in), static_cast<const unsigned char*>(packed),
      reinterpret_cast<const long long*>(bias), n_out, n_in, level, ctx->log_n, ctx->d_pi, ckks_wait_limit(ctx));
  return ckks_check_launch(fn);
}
