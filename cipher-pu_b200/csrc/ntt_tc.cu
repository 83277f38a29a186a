// ntt_tc.cu - the N = 2^12 negacyclic forward transform as two int8 matrix
// products on the 5th-generation tensor cores (tcgen05.mma kind::i8,
// accumulators in TMEM).  Same input, output order and results as ckks_ntt's
// forward negacyclic transform (ntt.cuh), which it is measured against.
//
// Four-step form, N = 64 x 64, input index j = j1 + 64 j2, output k = k1 + 64 k2:
//   A_k = sum_j a_j psi^(j (2k + 1))
//       = sum_j1 psi^(128 j1 k2) psi^(j1 (2 k1 + 1)) sum_j2 a_(j1 + 64 j2) psi^(64 j2 (2 k1 + 1))
//   step 1:  B[k1][j1] = sum_j2 F1[j2][k1] a[j1 + 64 j2],  F1 = psi^(64 j2 (2 k1 + 1))
//            (one 64-point negacyclic transform per j1)
//   twiddle: B'[j1][k1] = B[k1][j1] T[j1][k1],            T  = psi^(j1 (2 k1 + 1))
//   step 2:  A[k1 + 64 k2] = sum_j1 F2[j1][k2] B'[j1][k1], F2 = psi^(128 j1 k2)
// A_k is stored at the bit-reversed position 64 brv6(k1) + brv6(k2) = brv12(k),
// the evaluation order of the merged Cooley-Tukey transform.
//
// Exact products through byte limbs: residues x in [0, q) as 6 unsigned bytes
// x_a, matrix entries centred (|F| <= q / 2 < 2^46) as 6 balanced signed bytes
// f_b in [-128, 127].  The 128 MMA rows hold two limbs of the matrix at once
// (rows 0..63 limb b = p, rows 64..127 limb b = p + 3, p = 0, 1, 2), so the
// product of data limb a with row pair p belongs to accumulator range
// r = a + p: plane c = r in TMEM lanes 0..63 and c = r + 3 in lanes 64..127.
// 8 ranges x 32 columns (N = 32 positions per MMA) = 256 TMEM columns; a
// tile of 32 positions is 6 x 3 x 2 = 36 MMAs of 128 x 32 x 32, and
// |D_r| <= 3 * 64 * 255 * 128 < 2^23.
// Epilogue: S = sum_r D_r 256^r = lo + 2^32 hi with lo, hi exact integers
// below 2^48 in magnitude, so S = lo + hi [2^32]_q mod q is one FP64
// modular product (fmulmod, ntt.cuh); the upper lanes' sum is further
// multiplied by [2^24]_q and handed to the lower lanes' thread of the same
// row through shared memory.
//
// One CTA of 256 threads per limb-polynomial, two CTAs per SM (112 KB shared
// memory, 256 TMEM columns each; the exchange rows are XOR-swizzled, no padding): a 48 KB image of both matrices for the
// limb's prime arrives by one bulk asynchronous copy (no multicast), the
// polynomial is split into the step-1 operand image, and four tiles (step 1
// positions 0..31 / 32..63, step 2 likewise) each run 36 MMAs (one thread),
// a commit to an mbarrier (bounded wait) and the epilogue.  Every wait has an
// iteration limit; an expired wait drains the issued work (bounded), counts
// itself for ckks_device_status, frees TMEM and leaves the polynomial as it
// was.
#include <cstring>
#include <mutex>
#include <vector>

#include "ctx.hpp"
#include "dispatch.cuh"
#include "tmem.cuh"
#include "umma.cuh"
#include "profile.hpp"

namespace {

constexpr int NT_N = 4096;
constexpr int NT_THREADS = 256;
constexpr int NT_IMG = 128 * 64;            // one A image: 128 rows x 64 K bytes
constexpr int NT_PLANE = 64 * 64;           // one B plane: 64 rows x 64 K bytes
constexpr int NT_F_BYTES = 6 * NT_IMG;      // F2's 3 images, then F1's 3: 48 KB
// shared memory map (bytes)
constexpr int SM_F2 = 0;
constexpr int SM_F1 = 3 * NT_IMG;                      // 24 KB
constexpr int SM_B1 = 6 * NT_IMG;                      // 48 KB: step-1 operand (rows j1, K j2)
constexpr int SM_B2 = SM_B1 + 6 * NT_PLANE;            // 72 KB: step-2 operand (rows k1, K j1)
constexpr int SM_X = SM_B2 + 6 * NT_PLANE;             // 96 KB: upper lanes' partial sums
constexpr int SM_TOTAL = SM_X + 64 * 32 * 8;           // 112 KB: two CTAs per SM
constexpr int SM_OUT = SM_F1;  // output staging, 32 KB over F1 and B1 (both dead after step 1)
static_assert(SM_OUT + NT_N * 8 <= SM_B2, "output staging must not reach the step-2 operand");
constexpr int NT_TCOLS = 256;
// per-prime table: the 48 KB matrix image, T as (w, w / q) pairs, 4 constants
constexpr int NT_TAB_T = NT_F_BYTES;
constexpr int NT_TAB_C = NT_TAB_T + NT_N * 16;
constexpr int NT_TAB = NT_TAB_C + 64;

// byte offset of (row, k) in an operand image whose rows hold 64 K bytes
__host__ __device__ constexpr int nimg_off(int row, int k) {
  return (row >> 3) * 512 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15);
}

// instruction descriptor: D s32, A s8 (matrix limbs), B u8 (residue bytes),
// both K-major, N = 32, M = 128, dense
constexpr uint32_t kNtIdesc = (2u << 4) | (1u << 7) | (0u << 10) | ((uint32_t)(32 >> 3) << 17) |
                              ((uint32_t)(128 >> 4) << 24);

__device__ unsigned int g_ntt_tc_wait_expiries;

__device__ __forceinline__ void nt_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kNtIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ int brv6(int x) { return (int)(__brev((unsigned)x) >> 26); }

}  // namespace

__global__ void __launch_bounds__(NT_THREADS, 2)
    k_ntt_tc(u64* __restrict__ data, int n_limbs, int prime_begin, const PrimeInfo* __restrict__ pi,
             const unsigned char* __restrict__ tabs, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(8) unsigned long long bars[2];  // 0: matrix image landed, 1: MMA commits
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int prime = prime_begin + (int)(blockIdx.x % (unsigned)n_limbs);
  u64* poly = data + (size_t)blockIdx.x * NT_N;
  const unsigned char* tab = tabs + (size_t)prime * NT_TAB;
  const uint32_t bar_tab = s_u32(&bars[0]), bar_mma = s_u32(&bars[1]);

  if (warp == 0) tmem_alloc_warp(&tmem_slot, NT_TCOLS);
  if (tid == 32) {
    tc_mbar_init(bar_tab);
    tc_mbar_init(bar_mma);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tbase = tmem_slot;
  if (tid == 0) tc_bulk_load(s_u32(sm + SM_F2), tab, NT_F_BYTES, bar_tab);

  // step-1 operand: row j1, K = j2.  Lane l of warp w takes row 8 w + (l & 7)
  // and K groups 16 i + 4 (l >> 3) .. + 3, so each 4-byte image store of a
  // warp hits 32 distinct banks; the loads of 8 consecutive rows are 64-byte runs.
  {
    const int row = 8 * warp + (lane & 7);
    u64 x[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int u = 0; u < 4; ++u) x[i][u] = __ldcs(poly + row + 64 * (16 * i + 4 * (lane >> 3) + u));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      uint32_t pl[6];
      byte_planes(x[i], pl);
      const int off = nimg_off(row, 16 * i + 4 * (lane >> 3));
#pragma unroll
      for (int a = 0; a < 6; ++a) *reinterpret_cast<uint32_t*>(sm + SM_B1 + a * NT_PLANE + off) = pl[a];
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");

  const PrimeInfo P = pi[prime];
  const double* cst = reinterpret_cast<const double*>(tab + NT_TAB_C);
  const double c32 = cst[0], c32q = cst[1], c24 = cst[2], c24q = cst[3];
  const TwD* tw = reinterpret_cast<const TwD*>(tab + NT_TAB_T);
  double* xch = reinterpret_cast<double*>(sm + SM_X);
  u64* stage = reinterpret_cast<u64*>(sm + SM_OUT);

  const int q4 = warp & 3;              // TMEM lane quarter of this warp
  const int trow = 32 * q4 + lane;      // TMEM lane = MMA row
  const int row = trow & 63;            // k1 (step 1) or k2 (step 2)
  const bool upper = trow >= 64;        // holds planes r + 3
  const int cbase = 16 * (warp >> 2);   // this warp's 16 of the tile's 32 columns
  const uint32_t lane_addr = (uint32_t)(32 * q4) << 16;

  bool ok = true, tab_seen = false;
  int pending = -1;  // parity of a commit issued and not yet seen complete
#pragma unroll 1
  for (int t = 0; t < 4; ++t) {
    const int st = t >> 1, h = t & 1;
    bool expired = false;
    if (tid == 0 && t == 0) {
      expired = !tc_mbar_wait(bar_tab, 0, wait_limit);
      tab_seen = !expired;
    }
    tmem_fence_before_sync();
    if (__syncthreads_or(expired)) {
      ok = false;
      break;
    }
    tmem_fence_after_sync();
    if (tid == 0) {
      // A: the matrix's row-pair images; B: the 32 operand rows of this tile
      const uint64_t da = umma_desc(s_u32(sm + (st == 0 ? SM_F1 : SM_F2)), 128, 512);
      const uint64_t db = umma_desc(s_u32(sm + (st == 0 ? SM_B1 : SM_B2)) + 2048u * (uint32_t)h, 128, 512);
#pragma unroll
      for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            const int r = a + p;
            const bool first = ks == 0 && a == (r > 2 ? r - 2 : 0);  // first product of range r
            nt_mma(tbase + (uint32_t)(r * 32), da + (uint64_t)((p * NT_IMG + ks * 256) >> 4),
                   db + (uint64_t)((a * NT_PLANE + ks * 256) >> 4), first ? 0u : 1u);
          }
      tc_commit(bar_mma);
    }
    pending = t & 1;
    expired = !tc_mbar_wait(bar_mma, (uint32_t)pending, wait_limit);
    if (__syncthreads_or(expired)) {
      ok = false;
      break;
    }
    pending = -1;
    tmem_fence_after_sync();

    // epilogue part 1: every thread sums its lane's 8 ranges at its 16 columns
    long long lo[16], hi[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) lo[c] = hi[c] = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      int d[16];
      tmem_ld16_i32(tbase + lane_addr + (uint32_t)(r * 32 + cbase), d);
      const long long m = 1ll << (8 * (r & 3));
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        if (r < 4) lo[c] += (long long)d[c] * m;
        else hi[c] += (long long)d[c] * m;
      }
    }
    double s[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      s[c] = __dadd_rn(__ll2double_rn(lo[c]), fmulmod(__ll2double_rn(hi[c]), c32, c32q, P.qd));
      if (upper) xch[row * 32 + ((cbase + c) ^ (row & 31))] = fmulmod(s[c], c24, c24q, P.qd);
    }
    __syncthreads();
    // epilogue part 2: the lower lanes' threads finish their row
    if (!upper) {
#pragma unroll
      for (int c = 0; c < 16; ++c) s[c] = __dadd_rn(s[c], xch[row * 32 + ((cbase + c) ^ (row & 31))]);  // |s| < 2^49
      if (st == 0) {
        // B'[j1][k1] = B T, canonical, written as step-2 operand row k1, K = j1
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          u64 v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int j1 = 32 * h + cbase + 4 * g + u;
            const TwD w = ldtwd(tw + j1 * 64 + row);
            v[u] = d2canon(fmulmod(s[4 * g + u], w.w, w.wq, P.qd), P.qd, P.qinv_d);
          }
          uint32_t pl[6];
          byte_planes(v, pl);
          const int off = nimg_off(row, 32 * h + cbase + 4 * g);
#pragma unroll
          for (int a = 0; a < 6; ++a) *reinterpret_cast<uint32_t*>(sm + SM_B2 + a * NT_PLANE + off) = pl[a];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      } else {
        const int b2 = brv6(row);
#pragma unroll
        for (int c = 0; c < 16; ++c) stage[64 * brv6(32 * h + cbase + c) + b2] = d2canon(s[c], P.qd, P.qinv_d);
      }
    }
  }
  if (!ok) {
    // drain what may still be in flight (bounded), then count the expiry
    if (tid == 0) {
      atomicAdd(&g_ntt_tc_wait_expiries, 1u);
      if (!tab_seen && !tc_mbar_wait(bar_tab, 0, kTcDrainCycles)) atomicAdd(&g_ntt_tc_wait_expiries, 1u);
      if (pending >= 0 && !tc_mbar_wait(bar_mma, (uint32_t)pending, kTcDrainCycles))
        atomicAdd(&g_ntt_tc_wait_expiries, 1u);  // MMAs still running after the drain limit
    }
  }
  tmem_fence_before_sync();
  __syncthreads();
  if (ok) {
#pragma unroll
    for (int m = 0; m < NT_N / NT_THREADS; ++m) poly[tid + NT_THREADS * m] = stage[tid + NT_THREADS * m];
  }
  if (warp == 0) tmem_dealloc_warp(tbase, NT_TCOLS);
}

// ------------------------------------------------------------------ host side
namespace {
std::mutex g_ntt_tc_mu;

void balanced_bytes(long long v, signed char (&out)[6]) {
  for (int b = 0; b < 6; ++b) {
    long long d = v & 0xFF;
    if (d > 127) d -= 256;
    out[b] = (signed char)d;
    v = (v - d) / 256;
  }
}

// tables of every prime with a 2N-th root, built once per context
int ntt_tc_tables(ckks_ctx* ctx, const char* fn) {
  std::lock_guard<std::mutex> lock(g_ntt_tc_mu);
  if (ctx->d_ntt_tc) return CKKS_OK;
  std::vector<unsigned char> h((size_t)ctx->n_primes * NT_TAB, 0);
  for (int i = 0; i < ctx->n_primes; ++i) {
    if (!ctx->has_nega[i]) continue;
    const u64 q = ctx->primes[i], psi = ctx->psi[i];
    unsigned char* base = h.data() + (size_t)i * NT_TAB;
    std::vector<u64> pw(2 * NT_N);  // psi^e, e < 2N
    pw[0] = 1;
    for (int e = 1; e < 2 * NT_N; ++e) pw[e] = h_mulmod(pw[e - 1], psi, q);
    auto put = [&](int img_base, int m_row, int k, u64 v) {
      const long long c = v > q / 2 ? (long long)v - (long long)q : (long long)v;
      signed char d[6];
      balanced_bytes(c, d);
      for (int half = 0; half < 2; ++half)
        for (int pp = 0; pp < 3; ++pp)
          base[img_base + pp * NT_IMG + nimg_off(64 * half + m_row, k)] = (unsigned char)d[pp + 3 * half];
    };
    for (int m = 0; m < 64; ++m)
      for (int k = 0; k < 64; ++k) {
        put(SM_F2, m, k, pw[(128ull * k * m) % (2 * NT_N)]);             // F2[j1 = k][k2 = m]
        put(SM_F1, m, k, pw[(64ull * k * (2 * m + 1)) % (2 * NT_N)]);    // F1[j2 = k][k1 = m]
      }
    TwD* T = reinterpret_cast<TwD*>(base + NT_TAB_T);
    for (int j1 = 0; j1 < 64; ++j1)
      for (int k1 = 0; k1 < 64; ++k1) T[j1 * 64 + k1] = h_twd(pw[((u64)j1 * (2 * k1 + 1)) % (2 * NT_N)], q);
    double* cst = reinterpret_cast<double*>(base + NT_TAB_C);
    const u64 c32 = (1ull << 32) % q, c24 = (1ull << 24) % q;
    cst[0] = (double)c32;
    cst[1] = (double)c32 / (double)q;
    cst[2] = (double)c24;
    cst[3] = (double)c24 / (double)q;
  }
  unsigned char* d = nullptr;
  if (cudaError_t e = cudaMalloc(&d, h.size())) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  if (cudaError_t e = cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice)) {
    cudaFree(d);
    return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  }
  ctx->d_ntt_tc = d;
  return CKKS_OK;
}
}  // namespace

int ckks_ntt_tc_status_take(unsigned int* n) {
  cudaError_t e = cudaMemcpyFromSymbol(n, g_ntt_tc_wait_expiries, sizeof(*n));
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  if (*n) {
    const unsigned int zero = 0;
    e = cudaMemcpyToSymbol(g_ntt_tc_wait_expiries, &zero, sizeof(zero));
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  }
  return CKKS_OK;
}

extern "C" int ckks_ntt_tc(ckks_ctx* ctx, uint64_t* data, int n_polys, int prime_begin, int n_limbs,
                           void* stream) {
  ProfSpan span(CKKS_STAGE_OTHER, as_stream(stream), "ckks NTT (tensor cores)");
  const char* fn = "ckks_ntt_tc";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(ctx->log_n == 12, "%s: built for N = 2^12 only (context has N = 2^%d)", fn, ctx->log_n);
  CKKS_REQUIRE(prime_begin >= 0 && n_limbs >= 1 && prime_begin + n_limbs <= ctx->n_primes,
               "%s: limbs [%d, %d) outside the context's %d primes", fn, prime_begin, prime_begin + n_limbs,
               ctx->n_primes);
  CKKS_REQUIRE(n_polys >= 0, "%s: n_polys < 0", fn);
  for (int l = prime_begin; l < prime_begin + n_limbs; ++l)
    CKKS_REQUIRE(ctx->has_nega[l], "%s: prime %d has no 2N-th root; negacyclic transform unavailable", fn, l);
  if (n_polys == 0) return CKKS_OK;
  CKKS_REQUIRE(data != nullptr, "%s: data is NULL", fn);
  CKKS_REQUIRE((long long)n_polys * n_limbs <= 0x7FFFFFFFll, "%s: too many limb-polynomials", fn);
  if (int rc = ntt_tc_tables(ctx, fn)) return rc;
  if (cudaError_t e = ensure_smem(k_ntt_tc, SM_TOTAL))
    return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  k_ntt_tc<<<(unsigned)((long long)n_polys * n_limbs), NT_THREADS, SM_TOTAL, as_stream(stream)>>>(
      reinterpret_cast<u64*>(data), n_limbs, prime_begin, ctx->d_pi, ctx->d_ntt_tc, ckks_wait_limit(ctx));
  return ckks_check_launch(fn);
}
