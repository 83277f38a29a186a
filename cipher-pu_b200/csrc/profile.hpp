// profile.hpp - stage ids and the RAII span used by instrumented launches.
//
// A span always opens an NVTX range named after its stage (or the name
// given) around the host-side launch, so a profiler attached to the process
// (ncu --nvtx, Nsight Systems) attributes each kernel to its stage; with no
// tool attached an NVTX push / pop is a few nanoseconds.  When the library's
// own profiler is on (ckks_profile_enable), the span also records two CUDA
// events on the launching stream for ckks_profile_read.
#pragma once
#include <cuda_runtime.h>

#include "ctx.hpp"

enum {
  CKKS_STAGE_CM_TENSOR = 0,  // ct-mult: tensor product + d2 INTT
  CKKS_STAGE_CM_MODUP = 1,   // ct-mult: ModUp NTTs + key inner product
  CKKS_STAGE_CM_DOWN = 2,    // ct-mult: ModDown + rescale
  CKKS_STAGE_NTT = 3,        // standalone batched NTT
  CKKS_STAGE_OTHER = 4,
  CKKS_STAGE_CM_FUSED = 5,   // ct-mult: the one-cluster-per-pair kernel
  CKKS_STAGE_BATCH = 6,      // the persistent batch kernel
  CKKS_PROFILE_STAGES = 8
};

bool prof_on();

class ProfSpan {
 public:
  ProfSpan(int stage, cudaStream_t s, const char* nvtx_name = nullptr);
  ~ProfSpan();

 private:
  int stage_;
  cudaStream_t s_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
  bool active_ = false;
};
