// ctmul_host.cu - the batched ct-mult + relin + rescale on HOST buffers: the
// call a binding makes when its ciphertexts live in host memory (numpy arrays
// behind ctypes, a JVM direct buffer, a cgo slice).
//
// The batch is cut into chunks; chunk i runs on pipeline stream i mod 3 (the
// rotation continues from the previous call's last stream) as
// H2D(a, b) -> the three ct-mult kernels -> D2H(out), so the host->device copy
// of one chunk, the kernels of the previous one and the device->host copy of
// the one before that overlap (B200 has separate copy engines per direction).
// Each stream owns one slot of the caller's device workspace (inputs, output
// and ct-mult scratch of one chunk), so a slot is reused only after its
// previous chunk has left the stream.  The call returns when every output is
// in host memory.  Host buffers should be page-locked (cudaHostAlloc /
// torch pin_memory) for the copies to run asynchronously; pageable buffers
// give the same results with serialised copies.
//
// The _async entries enqueue the same pipeline and return at once; a later
// ckks_ct_mul_host_join(stream) makes the caller's stream wait for every
// chunk enqueued so far.  Back-to-back async calls keep the host->device copy
// engine busy across calls: the next call's first input copies run while the
// previous call's last chunks compute and copy back, which the blocking call
// cannot do (it drains the pipeline before returning).
#include <atomic>
#include <mutex>

#include "ctmul.hpp"

int ckks_launch_unpack48(uint64_t* out, const void* in, long long n, cudaStream_t st);
int ckks_launch_pack48(void* out, const uint64_t* in, long long n, cudaStream_t st);

namespace {

constexpr int kPipe = 3;
constexpr int kMaxDevices = 128;

struct Pipe {
  bool ready = false;
  cudaStream_t s[kPipe];
  cudaEvent_t start;
  cudaEvent_t done[kPipe];        // join points of the pipeline streams
  std::atomic<unsigned> next{0};  // stream of the next chunk: the rotation continues across calls
};

std::mutex g_pipe_mu;
Pipe g_pipe[kMaxDevices];

// Pipeline streams of the current device, created on first use and kept for
// the life of the process.
int pipe_for_device(Pipe** out, const char* fn) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: device %d beyond %d", fn, dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_pipe_mu);
  Pipe& p = g_pipe[dev];
  if (!p.ready) {
    for (int i = 0; i < kPipe && e == cudaSuccess; ++i)
      e = cudaStreamCreateWithFlags(&p.s[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.start, cudaEventDisableTiming);
    for (int i = 0; i < kPipe && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&p.done[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    p.ready = true;
  }
  *out = &p;
  return CKKS_OK;
}

struct Slot {
  size_t a_words, out_words, scratch_bytes, packed_bytes, total_bytes;
};

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// one stream's share of the workspace: inputs, output, ct-mult scratch and,
// for the packed wire format, the packed staging of both inputs and the output
Slot slot_shape(const ckks_ctx* ctx, int chunk, int level, bool packed) {
  Slot s;
  s.a_words = (size_t)chunk * 2 * level * ctx->n;
  s.out_words = (size_t)chunk * 2 * (level - 1) * ctx->n;
  s.scratch_bytes = ckks_ct_mul_scratch_bytes(ctx, chunk, level);
  s.packed_bytes = packed ? round256(6 * (2 * s.a_words + s.out_words)) : 0;
  s.total_bytes = (2 * s.a_words + s.out_words) * sizeof(uint64_t) + round256(s.scratch_bytes) + s.packed_bytes;
  return s;
}

}  // namespace

extern "C" size_t ckks_ct_mul_host_workspace_bytes(const ckks_ctx* ctx, int chunk, int level) {
  if (!ctx || chunk < 1 || level < 2) return 0;
  return (size_t)kPipe * slot_shape(ctx, chunk, level, false).total_bytes;
}

extern "C" size_t ckks_ct_mul_host48_workspace_bytes(const ckks_ctx* ctx, int chunk, int level) {
  if (!ctx || chunk < 1 || level < 2) return 0;
  return (size_t)kPipe * slot_shape(ctx, chunk, level, true).total_bytes;
}

static int host_pipeline(const ckks_ctx* ctx, void* out_host, const void* a_host, const void* b_host,
                         const uint64_t* key, int n_ct, int level, int chunk, void* workspace,
                         size_t workspace_bytes, void* stream, bool packed, bool wait, const char* fn) {
  CKKS_REQUIRE(ctx != nullptr, "%s: ctx is NULL", fn);
  CKKS_REQUIRE(n_ct >= 0, "%s: n_ct < 0", fn);
  CKKS_REQUIRE(chunk >= 1, "%s: chunk=%d must be >= 1", fn, chunk);
  CKKS_REQUIRE(level >= 2 && level <= ctx->n_q, "%s: level=%d outside [2, %d]", fn, level, ctx->n_q);
  if (n_ct == 0) return CKKS_OK;
  CKKS_REQUIRE(out_host && a_host && b_host && key && workspace, "%s: NULL pointer argument", fn);
  const Slot sl = slot_shape(ctx, chunk, level, packed);
  CKKS_REQUIRE(workspace_bytes >= (size_t)kPipe * sl.total_bytes,
               "%s: workspace of %zu bytes < %zu needed (ckks_ct_mul_host%s_workspace_bytes)", fn,
               workspace_bytes, (size_t)kPipe * sl.total_bytes, packed ? "48" : "");
  Pipe* p = nullptr;
  if (int rc = pipe_for_device(&p, fn)) return rc;
  // work queued earlier on the caller's stream (e.g. the key preparation)
  // comes first
  cudaError_t e = cudaEventRecord(p->start, as_stream(stream));
  for (int i = 0; i < kPipe && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(p->s[i], p->start, 0);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));

  const size_t in_ct = (size_t)2 * level * ctx->n;         // words per input ciphertext
  const size_t out_ct = (size_t)2 * (level - 1) * ctx->n;  // words per output ciphertext
  const size_t wb = packed ? 6 : sizeof(uint64_t);          // host bytes per word
  const unsigned char* ah = reinterpret_cast<const unsigned char*>(a_host);
  const unsigned char* bh = reinterpret_cast<const unsigned char*>(b_host);
  unsigned char* oh = reinterpret_cast<unsigned char*>(out_host);
  int rc = CKKS_OK;
  // chunk i of this call runs on stream (first + i) mod 3 with that stream's
  // workspace slot, so back-to-back stream-ordered calls spread over all three
  // streams even when a call has fewer chunks than streams
  const unsigned n_chunks = (unsigned)((n_ct + chunk - 1) / chunk);
  const unsigned first = p->next.fetch_add(n_chunks) % kPipe;
  for (int c0 = 0, i = 0; c0 < n_ct && rc == CKKS_OK; c0 += chunk, ++i) {
    const int m = n_ct - c0 < chunk ? n_ct - c0 : chunk;
    const unsigned si = (first + (unsigned)i) % kPipe;
    cudaStream_t st = p->s[si];
    unsigned char* base = reinterpret_cast<unsigned char*>(workspace) + (size_t)si * sl.total_bytes;
    uint64_t* da = reinterpret_cast<uint64_t*>(base);
    uint64_t* db = da + sl.a_words;
    uint64_t* dout = db + sl.a_words;
    void* scratch = dout + sl.out_words;
    unsigned char* pk = reinterpret_cast<unsigned char*>(scratch) + round256(sl.scratch_bytes);
    const size_t in_words = (size_t)m * in_ct;
    const size_t out_words = (size_t)m * out_ct;
    // packed staging: a at pk, b at pk + 6 a_words (16-byte aligned: a_words is a multiple of 8)
    void* sa = packed ? (void*)pk : (void*)da;
    void* sb = packed ? (void*)(pk + 6 * sl.a_words) : (void*)db;
    void* so = packed ? (void*)(pk + 12 * sl.a_words) : (void*)dout;
    e = cudaMemcpyAsync(sa, ah + (size_t)c0 * in_ct * wb, in_words * wb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sb, bh + (size_t)c0 * in_ct * wb, in_words * wb, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      rc = ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
      break;
    }
    if (packed) {
      rc = ckks_launch_unpack48(da, sa, (long long)in_words, st);
      if (rc == CKKS_OK) rc = ckks_launch_unpack48(db, sb, (long long)in_words, st);
      if (rc != CKKS_OK) break;
    }
    rc = ckks_ct_mul_launch(ctx, dout, da, db, key, m, level, scratch, sl.scratch_bytes, st, fn, 0, true);
    if (rc != CKKS_OK) break;
    if (packed) {
      rc = ckks_launch_pack48(so, dout, (long long)out_words, st);
      if (rc != CKKS_OK) break;
    }
    e = cudaMemcpyAsync(oh + (size_t)c0 * out_ct * wb, so, out_words * wb, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  }
  for (int i = 0; wait && i < kPipe; ++i) {
    const cudaError_t es = cudaStreamSynchronize(p->s[i]);
    if (es != cudaSuccess && rc == CKKS_OK)
      rc = ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(es));
  }
  return rc;
}

extern "C" int ckks_ct_mul_relin_rescale_host(const ckks_ctx* ctx, uint64_t* out_host,
                                              const uint64_t* a_host, const uint64_t* b_host,
                                              const uint64_t* key, int n_ct, int level, int chunk,
                                              void* workspace, size_t workspace_bytes,
                                              void* stream) {
  return host_pipeline(ctx, out_host, a_host, b_host, key, n_ct, level, chunk, workspace, workspace_bytes,
                       stream, false, true, "ckks_ct_mul_relin_rescale_host");
}

extern "C" int ckks_ct_mul_relin_rescale_host48(const ckks_ctx* ctx, void* out_host, const void* a_host,
                                                const void* b_host, const uint64_t* key, int n_ct,
                                                int level, int chunk, void* workspace,
                                                size_t workspace_bytes, void* stream) {
  return host_pipeline(ctx, out_host, a_host, b_host, key, n_ct, level, chunk, workspace, workspace_bytes,
                       stream, true, true, "ckks_ct_mul_relin_rescale_host48");
}

extern "C" int ckks_ct_mul_relin_rescale_host_async(const ckks_ctx* ctx, uint64_t* out_host,
                                                    const uint64_t* a_host, const uint64_t* b_host,
                                                    const uint64_t* key, int n_ct, int level, int chunk,
                                                    void* workspace, size_t workspace_bytes, void* stream) {
  return host_pipeline(ctx, out_host, a_host, b_host, key, n_ct, level, chunk, workspace, workspace_bytes,
                       stream, false, false, "ckks_ct_mul_relin_rescale_host_async");
}

extern "C" int ckks_ct_mul_relin_rescale_host48_async(const ckks_ctx* ctx, void* out_host, const void* a_host,
                                                      const void* b_host, const uint64_t* key, int n_ct,
                                                      int level, int chunk, void* workspace,
                                                      size_t workspace_bytes, void* stream) {
  return host_pipeline(ctx, out_host, a_host, b_host, key, n_ct, level, chunk, workspace, workspace_bytes,
                       stream, true, false, "ckks_ct_mul_relin_rescale_host48_async");
}

extern "C" int ckks_ct_mul_host_join(void* stream) {
  const char* fn = "ckks_ct_mul_host_join";
  Pipe* p = nullptr;
  if (int rc = pipe_for_device(&p, fn)) return rc;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < kPipe && e == cudaSuccess; ++i) {
    e = cudaEventRecord(p->done[i], p->s[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(as_stream(stream), p->done[i], 0);
  }
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  return CKKS_OK;
}
