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
int ckks_ct_mul_launch(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                       const uint64_t* ct_b, const uint64_t* key, int n_ct, int level,
                       void* scratch, size_t scratch_bytes, void* stream, const char* fn,
                       int max_split);
