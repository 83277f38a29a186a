// tmem.cuh - Blackwell Tensor Memory (TMEM) as per-thread storage.
//
// TMEM is 128 lanes x 512 columns of 32-bit cells per SM, allocated per CTA in
// power-of-two column counts (>= 32) by one warp (tcgen05.alloc) and returned
// before the CTA exits (tcgen05.dealloc).  Warp w of a CTA reaches lanes
// 32 (w mod 4) .. 32 (w mod 4) + 31 only; with the .32x32b shape thread i of
// the warp reads / writes lane 32 (w mod 4) + i, one 32-bit cell per column.
// So thread tid owns lane tid mod 128 of the column range the CTA gives its
// warp group (tid / 128): a private array of 32-bit cells next to the
// register file, used here for accumulators that must live across transforms.
//
// An address is (lane << 16) | column.  Loads and stores are asynchronous;
// each helper below waits for its own completion inside the same asm
// statement, so the compiler cannot use a loaded register early and a later
// load of the same cells sees the store.  They touch no memory the compiler
// tracks (no "memory" clobber); being volatile, they keep their order.
#pragma once
#include <cstdint>

__device__ __forceinline__ uint32_t tmem_smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Executed by ONE whole warp: allocate `ncols` columns (a power of two, >= 32);
// the base address is written to *slot (shared memory).  The CTA then gives
// up its permit to allocate again.
__device__ __forceinline__ void tmem_alloc_warp(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tmem_smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Executed by the same warp that allocated, after every thread's last access.
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// Order TMEM accesses (and the allocation) around a thread barrier.
__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// This thread's 8 doubles at columns [col, col + 16) of `taddr`'s lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, double (&v)[8]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __hiloint2double((int)r[2 * i + 1], (int)r[2 * i]);
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const double (&v)[8]) {
  uint32_t r[16];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    r[2 * i] = (uint32_t)__double2loint(v[i]);
    r[2 * i + 1] = (uint32_t)__double2hiint(v[i]);
  }
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15, %16};\n\t"
      "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
      "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]));
}

// Columns a CTA of `threads` threads needs for `cols_per_thread` 32-bit cells
// per thread: each group of 128 threads (4 warps, all 128 lanes) takes its
// own column range; rounded up to a power of two >= 32.
__host__ __device__ constexpr uint32_t tmem_cols_for(int threads, int cols_per_thread) {
  uint32_t c = (uint32_t)(((threads + 127) / 128) * cols_per_thread);
  uint32_t p = 32;
  while (p < c) p <<= 1;
  return p;
}
