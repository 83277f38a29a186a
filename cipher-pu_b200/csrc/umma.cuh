// umma.cuh - helpers for the kernels that drive the 5th-generation tensor
// cores directly (tcgen05.mma kind::i8 with TMEM accumulators): mbarrier
// waits with an iteration limit, bulk asynchronous copies (no multicast),
// shared-memory matrix descriptors for the K-major no-swizzle ("interleave")
// operand layout, commits, byte-limb splitting of residues and TMEM loads.
#pragma once
#include <cstdint>

#include "common.cuh"

// Internal linkage, as when each file defined its own: every kernel file
// that includes this header gets its private copy.
namespace {

__device__ __forceinline__ uint32_t s_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void tc_mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool tc_mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool tc_mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  if (tc_mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (!tc_mbar_test(bar, parity)) {
    if (clock64() - t0 > limit) return false;
    __nanosleep(20);
  }
  return true;
}
constexpr long long kTcDrainCycles = 4000000000ll;

// one bulk asynchronous copy global -> shared (16-byte aligned addresses, a
// multiple of 16 bytes), completing as transaction bytes on `bar`
__device__ __forceinline__ void tc_bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// shared-memory matrix descriptor: no swizzle, version 1 (sm_100)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
// Byte planes of four residues x[0..3] (< 2^48): p[a] holds byte a of x[t]
// in its byte t.  A 4 x 4 byte transpose of the low words (8 byte
// permutes) and a 4 x 2 one of the high words' two low bytes (4 more).
__device__ __forceinline__ void byte_planes(const u64 (&x)[4], uint32_t (&p)[6]) {
  const uint32_t l0 = (uint32_t)x[0], l1 = (uint32_t)x[1], l2 = (uint32_t)x[2], l3 = (uint32_t)x[3];
  const uint32_t h0 = (uint32_t)(x[0] >> 32), h1 = (uint32_t)(x[1] >> 32);
  const uint32_t h2 = (uint32_t)(x[2] >> 32), h3 = (uint32_t)(x[3] >> 32);
  const uint32_t t0 = __byte_perm(l0, l1, 0x5140), t1 = __byte_perm(l0, l1, 0x7362);  // (l0,l1) bytes 0,1 / 2,3
  const uint32_t t2 = __byte_perm(l2, l3, 0x5140), t3 = __byte_perm(l2, l3, 0x7362);
  p[0] = __byte_perm(t0, t2, 0x5410);
  p[1] = __byte_perm(t0, t2, 0x7632);
  p[2] = __byte_perm(t1, t3, 0x5410);
  p[3] = __byte_perm(t1, t3, 0x7632);
  const uint32_t u0 = __byte_perm(h0, h1, 0x5140), u2 = __byte_perm(h2, h3, 0x5140);
  p[4] = __byte_perm(u0, u2, 0x5410);
  p[5] = __byte_perm(u0, u2, 0x7632);
}

// 8 consecutive 32-bit accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld8_i32(uint32_t taddr, int (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = (int)r[i];
}

// 16 consecutive 32-bit accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld16_i32(uint32_t taddr, int (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int)r[i];
}

}  // namespace
