// profile.cu - optional per-kernel device timing of the multi-kernel entry
// points (CUDA events recorded on the launching stream around each kernel).
// Off by default; when on, each instrumented launch records two events and
// ckks_profile_read() resolves them (synchronising on those events only).
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "profile.hpp"

namespace {
struct Pending {
  int stage;
  cudaEvent_t a, b;
};
struct Totals {
  double ms = 0.0;
  long long launches = 0;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_free;
Totals g_tot[CKKS_PROFILE_STAGES];

cudaEvent_t take_event() {
  if (!g_free.empty()) {
    cudaEvent_t e = g_free.back();
    g_free.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

bool prof_on() { return g_on; }

// NVTX range names of the stages (index = stage id)
const char* const kStageNames[CKKS_PROFILE_STAGES] = {
    "ckks ct-mult: tensor product + d2 INTT", "ckks ct-mult: ModUp + key inner product",
    "ckks ct-mult: ModDown + rescale",       "ckks NTT",
    "ckks other",                            "ckks ct-mult: fused cluster kernel",
    "ckks batch: persistent kernel",         "ckks stage 7"};

ProfSpan::ProfSpan(int stage, cudaStream_t s, const char* nvtx_name) : stage_(stage), s_(s) {
  nvtxRangePushA(nvtx_name ? nvtx_name
                           : (stage >= 0 && stage < CKKS_PROFILE_STAGES ? kStageNames[stage] : "ckks"));
  if (!g_on) return;
  std::lock_guard<std::mutex> lk(g_mu);
  a_ = take_event();
  b_ = take_event();
  cudaEventRecord(a_, s_);
  active_ = true;
}

ProfSpan::~ProfSpan() {
  if (active_) {
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEventRecord(b_, s_);
    g_pending.push_back({stage_, a_, b_});
  }
  nvtxRangePop();
}

extern "C" int ckks_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_on = on != 0;
  return CKKS_OK;
}

extern "C" int ckks_profile_reset(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& p : g_pending) {
    cudaEventSynchronize(p.b);
    g_free.push_back(p.a);
    g_free.push_back(p.b);
  }
  g_pending.clear();
  for (auto& t : g_tot) t = Totals();
  return CKKS_OK;
}

extern "C" int ckks_profile_read(int stage, double* total_ms, long long* launches) {
  if (stage < 0 || stage >= CKKS_PROFILE_STAGES || !total_ms || !launches)
    return ckks_set_error(CKKS_EINVAL, "ckks_profile_read: bad stage %d", stage);
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& p : g_pending) {
    cudaEventSynchronize(p.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    g_tot[p.stage].ms += ms;
    g_tot[p.stage].launches += 1;
    g_free.push_back(p.a);
    g_free.push_back(p.b);
  }
  g_pending.clear();
  *total_ms = g_tot[stage].ms;
  *launches = g_tot[stage].launches;
  return CKKS_OK;
}
