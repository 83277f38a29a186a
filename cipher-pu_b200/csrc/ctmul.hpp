// ctmul.hpp - internal launcher of the batched ct-mult + relin + rescale,
// shared by the public entry points (device buffers, host buffers, static
// scratch).
#pragma once
#include "ctx.hpp"

// Enqueue the ct-mult of n_ct pairs on `stream` with caller-provided scratch.
// max_split bounds the concurrent sub-batches the call may fork onto the
// library's internal streams: 1 keeps every launch on `stream` and creates no
// CUDA stream or event (the allocation-free entry needs that); 0 = no bound
// (the context's tuning or the default decides).
//
// allow_fused: take the one-cluster-per-pair kernel (ctmul_fused.cu, no
// scratch) when ckks_ct_mul_fused_will_run says so; false keeps the
// three-kernel path that works through `scratch`.
int ckks_ct_mul_launch(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                       const uint64_t* ct_b, const uint64_t* key, int n_ct, int level,
                       void* scratch, size_t scratch_bytes, void* stream, const char* fn,
                       int max_split, bool allow_fused);

// Scratch bytes of the three-kernel path (the fused path needs none).
size_t ckks_ct_mul_scratch_bytes_3k(const ckks_ctx* ctx, int n_ct, int level);

// Whether the fused kernel is built for this shape (log N in [10, 13],
// level in [2, 7], one special prime).
bool ckks_ct_mul_fused_supported(const ckks_ctx* ctx, int level);

// Whether a ct-mult at this level takes the fused kernel: selected by
// CKKS_TUNE_CM_FUSED = 1, supported, and schedulable on the current device
// (cluster occupancy, checked once and cached).
bool ckks_ct_mul_fused_will_run(const ckks_ctx* ctx, int level);

// Enqueue the fused kernel (ctmul_fused.cu).  Returns CKKS_EUNSUPPORTED,
// without setting an error message, for a shape it is not built for.
int ckks_ct_mul_fused(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a, const uint64_t* ct_b,
                      const uint64_t* key, int n_ct, int level, void* stream, const char* fn);
