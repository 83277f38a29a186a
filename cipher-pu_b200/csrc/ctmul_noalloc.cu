// ctmul_noalloc.cu - the batched ct-mult + relin + rescale with its scratch in
// a fixed static device array, for callers that cannot allocate device memory.
//
// Who needs it: code that is handed only its input and output buffers and has
// no allocator of its own - e.g. a plugin called from a foreign runtime (JNI,
// cgo, a database UDF) whose host process owns all device memory through its
// own pool, or a serving loop whose memory pool has already reserved the GPU
// so that a fresh cudaMalloc would fail or stall the other streams while it
// synchronises the device.  Such a caller cannot provide the ~640 KB per
// ciphertext pair of scratch that ckks_ct_mul_relin_rescale expects.
//
// The scratch lives in g_ctmul_static_scratch below (CKKS_NOALLOC_SCRATCH_BYTES,
// declared in include/ckks_b200.h).  Every GPU that loads this library holds
// that array until the process exits.  In host code the symbol is only a
// host-side stand-in, never a device address, so the device address is
// fetched with cudaGetSymbolAddress once per device (with that device
// current) on the first call made on it, and cached.
#include <mutex>

#include "ctmul.hpp"
#include "profile.hpp"

static __device__ __align__(256) unsigned char g_ctmul_static_scratch[CKKS_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 128;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};
}  // namespace

extern "C" int ckks_ct_mul_relin_rescale_noalloc(const ckks_ctx* ctx, uint64_t* out,
                                                 const uint64_t* ct_a, const uint64_t* ct_b,
                                                 const uint64_t* key, int n_ct, int level,
                                                 void* stream) {
  const char* fn = "ckks_ct_mul_relin_rescale_noalloc";
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_ct >= 0, "%s: n_ct < 0", fn);
  CKKS_REQUIRE(level >= 2 && level <= ctx->n_q, "%s: level=%d outside [2, %d]", fn, level,
               ctx->n_q);
  // The optional profiler creates CUDA events; keep this path free of any
  // resource creation.
  CKKS_REQUIRE(!prof_on(), "%s: profiling is enabled (ckks_profile_enable); disable it first", fn);
  const size_t per_pair = ckks_ct_mul_scratch_bytes_3k(ctx, 1, level);
  const size_t need = ckks_ct_mul_scratch_bytes_3k(ctx, n_ct, level);
  CKKS_REQUIRE(need <= (size_t)CKKS_NOALLOC_SCRATCH_BYTES,
               "%s: %d pairs at N=%d, level %d need %zu scratch bytes, above the fixed static "
               "buffer of %zu bytes; pass at most %zu pairs per call",
               fn, n_ct, ctx->n, level, need, (size_t)CKKS_NOALLOC_SCRATCH_BYTES,
               per_pair ? (size_t)CKKS_NOALLOC_SCRATCH_BYTES / per_pair : (size_t)0);
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: cudaGetDevice: %s", fn, cudaGetErrorString(e));
  CKKS_REQUIRE(dev >= 0 && dev < kMaxDevices, "%s: device index %d unsupported", fn, dev);
  CKKS_REQUIRE(dev == ctx->device, "%s: context belongs to device %d but device %d is current", fn,
               ctx->device, dev);
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_ctmul_static_scratch);
      if (e != cudaSuccess || p == nullptr)
        return ckks_set_error(CKKS_ECUDA, "%s: cudaGetSymbolAddress of the static scratch: %s", fn,
                              cudaGetErrorString(e));
      g_noalloc_addr[dev] = p;
    }
    base = g_noalloc_addr[dev];
  }
  // Every scratch word is written by the first two kernels before it is read,
  // so the contents left by the previous call need no clearing.  max_split = 1:
  // the whole batch stays on the caller's stream as one sub-batch, whatever
  // the context's CKKS_TUNE_CM_SPLIT or the batch size, because concurrent
  // sub-batches run on internal streams and events that the library creates
  // on their first use.  allow_fused = false: this entry is the three-kernel
  // path with its scratch in the static array.
  return ckks_ct_mul_launch(ctx, out, ct_a, ct_b, key, n_ct, level, base,
                            (size_t)CKKS_NOALLOC_SCRATCH_BYTES, stream, fn, 1, false);
}
