// batch_persistent.cu - the batched uneven workload in ONE persistent launch:
// ct x ct + relinearisation + rescale and ct x pt + rescale operations of
// mixed ring dimension (N = 2^12, 2^13) and level, drained from a device
// work queue by as many CTAs as the GPU holds at once.
//
// Work units are the ones the per-shape kernels run one CTA at a time
// (ctmul_units.cuh): a ct x ct pair is `level` tensor units, `level + 1`
// ModUp units and 2 ModDown units; a ct x pt item is 2 units.  The host plan
// (ckks_batch_plan_create) lists every unit once, in an order where each
// unit comes after the units it depends on, and places a dependent stage a
// configurable number of units (the lag) after its producers so that by the
// time a CTA takes it, the producers have usually finished; ct x pt units,
// which depend on nothing, fill the tail.  The list is cut into slots: one
// N = 2^13 unit (radix 2^4: all 512 threads of the CTA), or two consecutive
// N = 2^12 units (radix 2^4: 256 threads each, run side by side by the two
// halves of the CTA on their own named barriers and shared-memory halves, as
// two CTAs of the per-shape kernels share an SM).  CTAs take slots in list
// order from one atomic ticket (the next ticket is fetched while the current
// slot runs).  That paired list couples the halves: both must finish before
// the CTA takes its next slot.  The phased list (an option) avoids it: the
// N = 2^13 units come first, one per whole-CTA slot; then every N = 2^12
// unit is a half slot of its own, and each half of each CTA takes half slots
// from a second ticket as soon as its previous unit is done.  Each ring
// size is scheduled on its own (no item spans both), so the dependency and
// no-deadlock arguments below hold in each phase.
//
// Dependencies are per-item counters: a tensor unit adds 1 to its pair's
// counter when its stores are done (every thread fences, the CTA syncs, one
// thread does a release add); a ModUp unit waits until that counter reaches
// `level`, a ModDown unit until the ModUp counter reaches level + 1 (one
// thread spins with acquire loads, then the CTA syncs and reads the
// intermediates through L2 with ld.global.cg).  The wait cannot deadlock: a
// CTA only takes tickets in increasing order and every dependency has a lower
// ticket, so the lowest unfinished ticket is always being worked on.
//
// Every wait is bounded by `wait_limit` SM cycles (a kernel argument).  On
// expiry the CTA counts the event in g_batch_wait_expiries (read and cleared
// by ckks_device_status), raises the launch's abort flag and returns; every
// other CTA sees the flag at its next wait or ticket and returns too.  The
// finished-unit counters then tell which outputs are complete
// (ckks_batch_plan_incomplete).  No unit holds TMEM or asynchronous copies,
// so returning early leaves nothing in flight.
//
// Reference counterpart: the time-multiplexed poly-mult instances of
// rtl/m4/e2e_ckks_mult_ctrl_m4.sv:368-482 (four multiplications interleaved
// on one datapath), here thousands of uneven operations over 148 SMs.
#include <algorithm>
#include <deque>
#include <vector>

#include "ctmul_units.cuh"
#include "dispatch.cuh"
#include "profile.hpp"

namespace {

constexpr int PB_THREADS = 512;  // one N = 2^13 unit at radix 2^4, or two N = 2^12 units
constexpr int PB_HALF = 256;     // threads of one N = 2^12 unit at radix 2^4
// shared memory of one N = 2^12 unit (the largest: ModUp / ModDown accumulators)
constexpr int PB_SM12_WORDS = NttShape<12, 4>::SMEM_WORDS + 2 * 4096;
constexpr int PB_SM13_WORDS = NttShape<13, 4>::SMEM_WORDS + 2 * 8192;
enum { PB_TENSOR = 0, PB_MODUP = 1, PB_DOWN = 2, PB_CTPT = 3 };
constexpr unsigned PB_NONE = 0xFFFFFFFFu;

struct PbBucket {
  int op;        // CKKS_BATCH_CT_CT or CKKS_BATCH_CT_PT
  int log_n;
  int level;
  int n_ct;
  int nq;        // the context's q-prime count (the special prime's index)
  int pt_stride; // ct x pt: 1 = one plaintext per ciphertext, 0 = shared
  const u64* a;
  const u64* b;
  u64* out;
  const double* key;
  CmScratch S;
  const PrimeInfo* pi;
  const TwD* tw;
  const TwPair* pinv;
  const TwPair* qtinv;
  unsigned* cnt;  // ct x ct: [3][n_ct] tensor done, ModUp done, finished; ct x pt: [n_ct] finished
};

// One work unit: x = bucket << 8 | stage << 6 | sub (limb, target prime or
// output polynomial), y = item.  A slot is one or two units (u[1].x =
// PB_NONE: one).
using PbJob = uint2;
struct PbSlot {
  PbJob u[2];
};

// The bucket table travels as a kernel parameter (constant bank): the units
// then read their descriptors' fields as operands instead of holding them in
// registers, which at 128 registers a thread would spill the N = 2^13 ModUp.
constexpr int PB_MAX_BUCKETS = 128;
struct PbTable {
  PbBucket b[PB_MAX_BUCKETS];
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned* p) {
  return *reinterpret_cast<const volatile unsigned*>(p);
}

}  // namespace

__device__ unsigned int g_batch_wait_expiries;

// Thread 0: spin until *cnt >= target, the launch aborts, or `limit` cycles
// pass (then count the expiry and raise the abort flag).  True when met.
__device__ __noinline__ bool pb_wait(const unsigned* cnt, unsigned target, unsigned* abort_flag,
                                     long long limit) {
  const long long t0 = clock64();
  unsigned ns = 32;
  for (;;) {
    if (ld_acquire_u32(cnt) >= target) return true;
    if (ld_volatile_u32(abort_flag)) return false;
    if (clock64() - t0 > limit) {
      atomicAdd(&g_batch_wait_expiries, 1u);
      atomicExch(abort_flag, 1u);
      return false;
    }
    __nanosleep(ns);
    ns = ns < 512 ? 2 * ns : ns;
  }
}

template <int LOGN, int K>
__device__ __forceinline__ void pb_run_unit(const PbBucket& B, int stage, int sub, long long item, u64* sm,
                                            int tid) {
  switch (stage) {
    case PB_TENSOR:
      cm_tensor_unit<LOGN, K>(B.a, B.b, B.S, B.level, B.pi, B.tw, B.n_ct, (long long)sub * B.n_ct + item, sm, tid);
      break;
    case PB_MODUP:
      cm_modup_unit<LOGN, K, true>(B.S, B.key, B.level, B.nq, B.pi, B.tw, B.n_ct,
                                   (long long)(B.level - sub) * B.n_ct + item, sm, tid);
      break;
    case PB_DOWN:
      cm_down_unit<LOGN, K, true>(B.S, B.out, B.level, B.nq, B.pi, B.tw, B.pinv, B.qtinv, 2 * item + sub, sm, tid);
      break;
    default:
      ctpt_unit<LOGN, K>(B.out, B.a, B.b, B.pt_stride, B.level, B.pi, B.tw, B.qtinv, B.nq, item, sub, sm, tid);
      break;
  }
}

// One unit on one thread group (the whole CTA for N = 2^13, a half for
// 2^12; tid = the thread's index in its group, grp = the group): wait for its
// inputs if it has any, run it, publish it.  False when the wait gave up.
template <int LOGN, int K>
__device__ __forceinline__ void pb_unit(const PbTable& tab, PbJob jb, u64* sm, int tid, int grp, unsigned* ctl,
                                        long long wait_limit, int unmet_bucket, int* s_ok) {
  constexpr int T = NttShape<LOGN, K>::T;
  const int bi = (int)(jb.x >> 8), stage = (int)(jb.x >> 6) & 3, sub = (int)(jb.x & 63);
  const long long item = jb.y;
  const PbBucket& B = tab.b[bi];
  const int n_ct = B.n_ct;
  if (stage == PB_MODUP || stage == PB_DOWN) {
    if (tid == 0) {
      const unsigned* c = stage == PB_MODUP ? B.cnt + item : B.cnt + n_ct + item;
      unsigned target = stage == PB_MODUP ? (unsigned)B.level : (unsigned)B.level + 1;
      if (stage == PB_MODUP && bi == unmet_bucket && item == 0) target += 1;
      s_ok[grp] = pb_wait(c, target, ctl + 2, wait_limit);
    }
    group_sync<T>();
    if (!s_ok[grp]) return;
  }
  pb_run_unit<LOGN, K>(B, stage, sub, item, sm, tid);
  // publish: every thread's stores, then one release add for the group
  __threadfence();
  group_sync<T>();
  if (tid == 0) {
    unsigned* c = stage == PB_TENSOR ? B.cnt + item
                  : stage == PB_MODUP ? B.cnt + n_ct + item
                  : stage == PB_DOWN  ? B.cnt + 2 * (size_t)n_ct + item
                                      : B.cnt + item;
    red_release_add(c, 1u);
  }
}

// ctl[0..1]: the 64-bit ticket of the whole-CTA slots, ctl[2]: the abort
// flag, ctl[4..5]: the 64-bit ticket of the half slots (all zeroed before
// every launch).
// slots[0, n_slots): whole-CTA slots (one N = 2^13 unit, or in the paired
// list two N = 2^12 units side by side); slots[n_slots, n_slots + n_half):
// half slots, one N = 2^12 unit each, which each 256-thread half of every CTA
// takes from its own ticket once the CTA has run out of whole-CTA slots.
// unmet_bucket >= 0 is a test hook: the ModUp units of item 0 of that
// bucket wait for one tensor unit more than exist, so their wait can only
// end by its limit.
template <int MAXLOGN>
__global__ void __launch_bounds__(PB_THREADS, 1)
    k_batch_persistent(const __grid_constant__ PbTable tab, const PbSlot* __restrict__ slots, long long n_slots,
                       unsigned* ctl, long long wait_limit, int unmet_bucket) {
  extern __shared__ u64 sm[];
  __shared__ long long s_ticket;
  __shared__ int s_ok[2];
  const int tid = threadIdx.x;
  unsigned long long next = 0;
  if (tid == 0) next = atomicAdd(reinterpret_cast<unsigned long long*>(ctl), 1ull);
  for (;;) {
    if (tid == 0) {
      const unsigned long long t = next;
      const bool go = (long long)t < n_slots && !ld_volatile_u32(ctl + 2);
      // fetch the following ticket now; it is used once this slot is done
      if (go) next = atomicAdd(reinterpret_cast<unsigned long long*>(ctl), 1ull);
      s_ticket = go ? (long long)t : -1;
    }
    __syncthreads();
    const long long t = s_ticket;
    if (t < 0) return;
    const PbJob j0 = slots[t].u[0];
    bool big = false;
    if constexpr (MAXLOGN >= 13) big = tab.b[j0.x >> 8].log_n == 13;
    if (big) {
      if constexpr (MAXLOGN >= 13) pb_unit<13, 4>(tab, j0, sm, tid, 0, ctl, wait_limit, unmet_bucket, s_ok);
    } else {
      const int h = tid / PB_HALF;  // uniform within each half
      const PbJob jh = slots[t].u[h];
      if (jh.x != PB_NONE)
        pb_unit<12, 4>(tab, jh, sm + h * PB_SM12_WORDS, tid % PB_HALF, h, ctl, wait_limit, unmet_bucket, s_ok);
    }
    __syncthreads();  // both halves done: the shared memory is free for the next slot
  }
}

// The phased list: slots[0, n_whole) are N = 2^13 units, one per whole-CTA
// slot; slots[n_whole, n_whole + n_half) are N = 2^12 units, which each
// 256-thread half takes from the second ticket (ctl[4..5]) on its own once
// the CTA has run out of whole-CTA slots (its own named barrier and
// shared-memory half from then on).  One call site per unit shape.
template <int MAXLOGN>
__global__ void __launch_bounds__(PB_THREADS, 1)
    k_batch_phased(const __grid_constant__ PbTable tab, const PbSlot* __restrict__ slots, long long n_whole,
                   long long n_half, unsigned* ctl, long long wait_limit, int unmet_bucket) {
  extern __shared__ u64 sm[];
  __shared__ long long s_whole;     // phase 1 ticket (whole CTA)
  __shared__ long long s_half[2];   // phase 2 tickets (one per half)
  __shared__ int s_ok[2];
  const int tid = threadIdx.x;
  if constexpr (MAXLOGN >= 13) {
    unsigned long long next = 0;
    if (tid == 0 && n_whole > 0) next = atomicAdd(reinterpret_cast<unsigned long long*>(ctl), 1ull);
    for (;;) {
      if (tid == 0) {
        const unsigned long long t = next;
        const bool go = n_whole > 0 && (long long)t < n_whole && !ld_volatile_u32(ctl + 2);
        if (go) next = atomicAdd(reinterpret_cast<unsigned long long*>(ctl), 1ull);
        s_whole = go ? (long long)t : -1;
      }
      __syncthreads();
      const long long t = s_whole;
      if (t < 0) break;
      pb_unit<13, 4>(tab, slots[t].u[0], sm, tid, 0, ctl, wait_limit, unmet_bucket, s_ok);
      __syncthreads();  // the CTA's shared memory is free for the next unit
    }
  }
  const int h = tid / PB_HALF, ht = tid % PB_HALF;  // h is uniform within each half
  for (;;) {
    if (ht == 0) {
      const bool live = !ld_volatile_u32(ctl + 2);
      const unsigned long long t = live ? atomicAdd(reinterpret_cast<unsigned long long*>(ctl + 4), 1ull) : 0ull;
      s_half[h] = live && (long long)t < n_half ? (long long)t : -1;
    }
    group_sync<PB_HALF>();
    const long long t = s_half[h];
    if (t < 0) return;
    pb_unit<12, 4>(tab, slots[n_whole + t].u[0], sm + h * PB_SM12_WORDS, ht, h, ctl, wait_limit, unmet_bucket, s_ok);
    group_sync<PB_HALF>();  // the half's shared memory and ticket word are free again
  }
}

// Expiries of the persistent batch kernel's waits, read and cleared by
// ckks_device_status.
int ckks_batch_status_take(unsigned* n) {
  cudaError_t e = cudaMemcpyFromSymbol(n, g_batch_wait_expiries, sizeof(*n));
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  if (*n) {
    const unsigned zero = 0;
    e = cudaMemcpyToSymbol(g_batch_wait_expiries, &zero, sizeof(zero));
    if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "ckks_device_status: %s", cudaGetErrorString(e));
  }
  return CKKS_OK;
}

// ---------------------------------------------------------------- host plan
struct ckks_batch_plan {
  int device = 0;
  int max_log_n = 12;
  int grid = 0;
  int smem = 0;
  long long n_units = 0;
  long long n_slots = 0;   // paired list (the default): whole-CTA slots
  long long n_whole = 0;   // phased list: N = 2^13 whole-CTA slots, then
  long long n_half = 0;    // N = 2^12 half slots (stored after the paired list)
  int n_buckets = 0;
  unsigned char* mem = nullptr;  // one device allocation
  size_t mem_bytes = 0;
  size_t zero_bytes = 0;         // ctl + counters, at the start of mem
  unsigned* ctl = nullptr;
  PbSlot* d_slots = nullptr;
  std::vector<PbBucket> h_buckets;
  PbTable* table = nullptr;      // host copy passed at every launch
  std::vector<size_t> cnt_off;   // per bucket, in counters
  std::vector<unsigned> h_cnt;
  size_t n_cnt = 0;
};

namespace {

template <int MAXLOGN>
int pb_launch(ckks_batch_plan* p, bool paired, long long wait_limit, int unmet_bucket, cudaStream_t st) {
  if (paired)
    k_batch_persistent<MAXLOGN><<<p->grid, PB_THREADS, p->smem, st>>>(*p->table, p->d_slots, p->n_slots, p->ctl,
                                                                     wait_limit, unmet_bucket);
  else
    k_batch_phased<MAXLOGN><<<p->grid, PB_THREADS, p->smem, st>>>(
        *p->table, p->d_slots + p->n_slots, p->n_whole, p->n_half, p->ctl, wait_limit, unmet_bucket);
  return ckks_check_launch("ckks_batch_plan_run");
}

template <typename KernelT>
cudaError_t pb_raise_smem(KernelT k, int smem) {
  // raise the kernel's dynamic shared-memory cap, never lower it: plans of
  // other shapes may launch the same kernel with more
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, k);
  if (e == cudaSuccess && smem > fa.maxDynamicSharedSizeBytes)
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return e;
}

template <int MAXLOGN>
int pb_configure(ckks_batch_plan* p, const char* fn) {
  auto k = k_batch_persistent<MAXLOGN>;
  auto kp = k_batch_phased<MAXLOGN>;
  cudaError_t e0 = pb_raise_smem(k, p->smem);
  if (e0 == cudaSuccess) e0 = pb_raise_smem(kp, p->smem);
  if (e0 != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e0));
  int per_sm = 0, per_sm_p = 0, n_sm = 0;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, p->device);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, PB_THREADS, p->smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_p, kp, PB_THREADS, p->smem);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  per_sm = std::min(per_sm, per_sm_p);
  if (per_sm < 1)
    return ckks_set_error(CKKS_EUNSUPPORTED, "%s: the persistent kernel does not fit on an SM with %d B of shared memory",
                          fn, p->smem);
  p->grid = n_sm * per_sm;
  return CKKS_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// ---------------------------------------------------------------- the work list
// A greedy list schedule.  A ct x ct pair's ModUp units go in once `lag`
// units have been listed after its last tensor unit, its ModDown units `lag`
// after its last ModUp unit; otherwise the next pairs' tensor units go in
// (pairs of the costliest buckets first, two at a time), then ct x pt
// units; with nothing else left, a pending stage goes in early.  Every unit is listed once and
// after the units it depends on.  jobs must hold sum(n_ct (2 level + 3)) +
// sum(2 n_ct) entries (ct x ct, ct x pt buckets).
static void pb_schedule(int n_buckets, const int* op, const int* n_ct, const int* level, const double* cost,
                        long long lag, PbJob* jobs) {
  long long pos = 0;
  auto job = [](int b, int stage, int sub, long long item) {
    return PbJob{(unsigned)b << 8 | (unsigned)stage << 6 | (unsigned)sub, (unsigned)item};
  };
  std::vector<int> cm_order, pt_order;
  for (int b = 0; b < n_buckets; ++b) (op[b] == CKKS_BATCH_CT_CT ? cm_order : pt_order).push_back(b);
  std::stable_sort(cm_order.begin(), cm_order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  std::stable_sort(pt_order.begin(), pt_order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  long long total = 0;
  for (int b = 0; b < n_buckets; ++b) total += (long long)n_ct[b] * (op[b] == CKKS_BATCH_CT_CT ? 2 * level[b] + 3 : 2);
  // Pairs go in two at a time (items `item` and item + 1 of one bucket when
  // n_items = 2), their units interleaved, so consecutive units have the same
  // stage and length: two of them share a slot without one half idling.
  struct Pending {
    long long ready;
    int b, stage;
    long long item;
    int n_items;
  };
  std::deque<Pending> pend;
  size_t cb = 0, pb = 0;
  long long ci = 0, pi = 0;
  auto emit_pending = [&]() {
    const Pending q = pend.front();
    pend.pop_front();
    if (q.stage == PB_MODUP) {
      for (int ti = level[q.b]; ti >= 0; --ti)  // special prime first
        for (int i = 0; i < q.n_items; ++i) jobs[pos++] = job(q.b, PB_MODUP, ti, q.item + i);
      pend.push_back({pos + lag, q.b, PB_DOWN, q.item, q.n_items});
    } else {
      for (int k = 0; k < 2; ++k)
        for (int i = 0; i < q.n_items; ++i) jobs[pos++] = job(q.b, PB_DOWN, k, q.item + i);
    }
  };
  while (pos < total) {
    while (cb < cm_order.size() && ci >= n_ct[cm_order[cb]]) ++cb, ci = 0;
    while (pb < pt_order.size() && pi >= n_ct[pt_order[pb]]) ++pb, pi = 0;
    if (!pend.empty() && pend.front().ready <= pos) {
      emit_pending();
    } else if (cb < cm_order.size()) {
      const int b = cm_order[cb];
      const int m = ci + 1 < n_ct[b] ? 2 : 1;
      for (int j = 0; j < level[b]; ++j)
        for (int i = 0; i < m; ++i) jobs[pos++] = job(b, PB_TENSOR, j, ci + i);
      pend.push_back({pos + lag, b, PB_MODUP, ci, m});
      ci += m;
    } else if (pb < pt_order.size()) {
      const int b = pt_order[pb];
      for (int k = 0; k < 2; ++k) jobs[pos++] = job(b, PB_CTPT, k, pi);
      ++pi;
    } else {
      emit_pending();
    }
  }
}

// Cut the unit list into slots: an N = 2^13 unit alone; N = 2^12 units two
// by two in list order (a 2^12 unit waiting for its partner may be passed by
// 2^13 slots: it only moves later, after its own producers).  Returns the
// slot count; slots must hold n_units entries.
static long long pb_slots(const PbJob* jobs, long long n_units, const int* log_n, PbSlot* slots) {
  long long ns = 0;
  long long pending = -1;
  for (long long i = 0; i < n_units; ++i) {
    if (log_n[jobs[i].x >> 8] == 13) {
      slots[ns++] = PbSlot{{jobs[i], PbJob{PB_NONE, 0}}};
    } else if (pending >= 0) {
      slots[ns++] = PbSlot{{jobs[pending], jobs[i]}};
      pending = -1;
    } else {
      pending = i;
    }
  }
  if (pending >= 0) slots[ns++] = PbSlot{{jobs[pending], PbJob{PB_NONE, 0}}};
  return ns;
}

// The phased list: the N = 2^13 buckets scheduled alone, one unit per
// whole-CTA slot, then the N = 2^12 buckets scheduled alone, one unit per
// half slot (u[1] = none).  Returns the whole-CTA slot count; *n_half gets
// the half-slot count.  slots must hold every unit.
static long long pb_phased(int n_buckets, const int* op, const int* n_ct, const int* level, const int* log_n,
                           const double* cost, long long lag_whole, long long lag_half, PbSlot* slots,
                           long long* n_half) {
  std::vector<int> c13(n_buckets), c12(n_buckets);
  long long t13 = 0, t12 = 0;
  for (int b = 0; b < n_buckets; ++b) {
    const long long u = (long long)n_ct[b] * (op[b] == CKKS_BATCH_CT_CT ? 2 * level[b] + 3 : 2);
    c13[b] = log_n[b] == 13 ? n_ct[b] : 0;
    c12[b] = log_n[b] == 13 ? 0 : n_ct[b];
    (log_n[b] == 13 ? t13 : t12) += u;
  }
  std::vector<PbJob> jobs((size_t)std::max(t13, t12));
  pb_schedule(n_buckets, op, c13.data(), level, cost, lag_whole, jobs.data());
  for (long long i = 0; i < t13; ++i) slots[i] = PbSlot{{jobs[i], PbJob{PB_NONE, 0}}};
  pb_schedule(n_buckets, op, c12.data(), level, cost, lag_half, jobs.data());
  for (long long i = 0; i < t12; ++i) slots[t13 + i] = PbSlot{{jobs[i], PbJob{PB_NONE, 0}}};
  *n_half = t12;
  return t13;
}

// The work list on the host alone (no device, no context): slots gets 4 x
// uint32 per slot, two units (bucket << 8 | stage << 6 | sub, item) with
// stage 0 tensor, 1 ModUp, 2 ModDown, 3 ct x pt, the second 0xFFFFFFFF, 0 in
// a slot of one unit.  n_slots (in/out): capacity in (at least the number of
// units), slots listed out.  `cost` ranks the buckets (costliest first); `lag`
// in units.
extern "C" int ckks_batch_schedule(int n_buckets, const int* op, const int* n_ct, const int* level,
                                   const int* log_n, const double* cost, long long lag, uint32_t* slots,
                                   long long* n_slots) {
  const char* fn = "ckks_batch_schedule";
  CKKS_REQUIRE(n_slots != nullptr, "%s: n_slots is NULL", fn);
  CKKS_REQUIRE(n_buckets >= 0 && n_buckets <= PB_MAX_BUCKETS, "%s: n_buckets=%d outside [0, %d]", fn, n_buckets,
               PB_MAX_BUCKETS);
  CKKS_REQUIRE(n_buckets == 0 || (op && n_ct && level && log_n && cost), "%s: NULL pointer argument", fn);
  CKKS_REQUIRE(lag >= 0, "%s: lag < 0", fn);
  long long total = 0;
  for (int b = 0; b < n_buckets; ++b) {
    CKKS_REQUIRE(op[b] == CKKS_BATCH_CT_CT || op[b] == CKKS_BATCH_CT_PT, "%s: bucket %d: op=%d", fn, b, op[b]);
    CKKS_REQUIRE(n_ct[b] >= 0 && level[b] >= 2 && level[b] <= 62, "%s: bucket %d: n_ct=%d level=%d", fn, b, n_ct[b],
                 level[b]);
    CKKS_REQUIRE(log_n[b] == 12 || log_n[b] == 13, "%s: bucket %d: log_n=%d (12 or 13)", fn, b, log_n[b]);
    total += (long long)n_ct[b] * (op[b] == CKKS_BATCH_CT_CT ? 2 * level[b] + 3 : 2);
  }
  CKKS_REQUIRE(slots != nullptr || total == 0, "%s: slots is NULL", fn);
  CKKS_REQUIRE(*n_slots >= total, "%s: capacity %lld < %lld units", fn, *n_slots, total);
  std::vector<PbJob> jobs((size_t)total);
  pb_schedule(n_buckets, op, n_ct, level, cost, lag, jobs.data());
  *n_slots = pb_slots(jobs.data(), total, log_n, reinterpret_cast<PbSlot*>(slots));
  return CKKS_OK;
}

// The phased list on the host alone: *n_whole whole-CTA slots (one
// N = 2^13 unit each, dependent stages lag units apart), then the half slots
// (one N = 2^12 unit each, 2 lag units apart: two halves per CTA); the slot
// format of ckks_batch_schedule, every second unit (0xFFFFFFFF, 0).
extern "C" int ckks_batch_schedule_phased(int n_buckets, const int* op, const int* n_ct, const int* level,
                                          const int* log_n, const double* cost, long long lag, uint32_t* slots,
                                          long long* n_slots, long long* n_whole) {
  const char* fn = "ckks_batch_schedule_phased";
  CKKS_REQUIRE(n_slots != nullptr && n_whole != nullptr, "%s: NULL count argument", fn);
  CKKS_REQUIRE(n_buckets >= 0 && n_buckets <= PB_MAX_BUCKETS, "%s: n_buckets=%d outside [0, %d]", fn, n_buckets,
               PB_MAX_BUCKETS);
  CKKS_REQUIRE(n_buckets == 0 || (op && n_ct && level && log_n && cost), "%s: NULL pointer argument", fn);
  CKKS_REQUIRE(lag >= 0, "%s: lag < 0", fn);
  long long total = 0;
  for (int b = 0; b < n_buckets; ++b) {
    CKKS_REQUIRE(op[b] == CKKS_BATCH_CT_CT || op[b] == CKKS_BATCH_CT_PT, "%s: bucket %d: op=%d", fn, b, op[b]);
    CKKS_REQUIRE(n_ct[b] >= 0 && level[b] >= 2 && level[b] <= 62, "%s: bucket %d: n_ct=%d level=%d", fn, b, n_ct[b],
                 level[b]);
    CKKS_REQUIRE(log_n[b] == 12 || log_n[b] == 13, "%s: bucket %d: log_n=%d (12 or 13)", fn, b, log_n[b]);
    total += (long long)n_ct[b] * (op[b] == CKKS_BATCH_CT_CT ? 2 * level[b] + 3 : 2);
  }
  CKKS_REQUIRE(slots != nullptr || total == 0, "%s: slots is NULL", fn);
  CKKS_REQUIRE(*n_slots >= total, "%s: capacity %lld < %lld units", fn, *n_slots, total);
  long long n_half = 0;
  *n_whole = pb_phased(n_buckets, op, n_ct, level, log_n, cost, lag, 2 * lag, reinterpret_cast<PbSlot*>(slots),
                       &n_half);
  *n_slots = *n_whole + n_half;
  return CKKS_OK;
}

extern "C" int ckks_batch_plan_create(const ckks_batch_bucket* buckets, int n_buckets, int lag_percent,
                                      ckks_batch_plan** out) {
  const char* fn = "ckks_batch_plan_create";
  CKKS_REQUIRE(out != nullptr, "%s: out is NULL", fn);
  *out = nullptr;
  CKKS_REQUIRE(n_buckets >= 0 && n_buckets <= PB_MAX_BUCKETS, "%s: n_buckets=%d outside [0, %d]", fn, n_buckets,
               PB_MAX_BUCKETS);
  CKKS_REQUIRE(n_buckets == 0 || buckets != nullptr, "%s: buckets is NULL", fn);
  CKKS_REQUIRE(lag_percent >= 0 && lag_percent <= 10000, "%s: lag_percent=%d outside [0, 10000]", fn, lag_percent);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: no current device", fn);
  auto p = new ckks_batch_plan();
  p->device = dev;
  p->n_buckets = n_buckets;
  auto fail = [&](int rc) {
    if (p->mem) cudaFree(p->mem);
    delete p->table;
    delete p;
    return rc;
  };
  // ---- validate and size
  size_t scratch_words = 0;
  long long n_units = 0;
  int smem = 0;
  for (int b = 0; b < n_buckets; ++b) {
    const ckks_batch_bucket& B = buckets[b];
    const ckks_ctx* ctx = B.ctx;
    if (!ctx) return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: ctx is NULL", fn, b));
    if (ctx->device != dev)
      return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: context of device %d, current device %d", fn, b,
                                 ctx->device, dev));
    if (ctx->log_n != 12 && ctx->log_n != 13)
      return fail(ckks_set_error(CKKS_EUNSUPPORTED, "%s: bucket %d: log_n=%d (built for 12 and 13)", fn, b,
                                 ctx->log_n));
    if (B.op != CKKS_BATCH_CT_CT && B.op != CKKS_BATCH_CT_PT)
      return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: op=%d", fn, b, B.op));
    if (B.n_ct < 0 || B.n_ct >= (1 << 30))
      return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: n_ct=%d", fn, b, B.n_ct));
    if (B.level < 2 || B.level > ctx->n_q)
      return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: level=%d outside [2, %d]", fn, b, B.level, ctx->n_q));
    if (B.n_ct > 0 && !(B.a && B.b && B.out && (B.op == CKKS_BATCH_CT_PT || B.key)))
      return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: NULL pointer argument", fn, b));
    for (int i = 0; i < ctx->n_primes; ++i)
      if (!ctx->has_nega[i])
        return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: prime %d has no 2N-th root", fn, b, i));
    const int N = ctx->n;
    // an N = 2^13 unit uses the whole CTA's shared memory; 2^12 units run two
    // side by side, each in a fixed half of PB_SM12_WORDS
    smem = std::max(smem, ctx->log_n == 13 ? PB_SM13_WORDS * 8 : 2 * PB_SM12_WORDS * 8);
    if (B.op == CKKS_BATCH_CT_CT) {
      if (ctx->n_special != 1)
        return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: context needs exactly one special prime", fn, b));
      u64 pmin = ~0ull, pmax = 0;
      for (int i = 0; i < ctx->n_primes; ++i) {
        pmin = std::min(pmin, ctx->primes[i]);
        pmax = std::max(pmax, ctx->primes[i]);
      }
      if (!(pmax < 2 * pmin))
        return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: primes must satisfy max < 2 min", fn, b));
      scratch_words += (size_t)B.n_ct * (6 * B.level + 2) * N;
      n_units += (long long)B.n_ct * (2 * B.level + 3);
    } else {
      for (int i = 0; i < B.level - 1; ++i)
        if (!(ctx->primes[B.level - 1] < 2 * ctx->primes[i]))
          return fail(ckks_set_error(CKKS_EINVAL, "%s: bucket %d: q_%d must be < 2 q_%d", fn, b, B.level - 1, i));
      n_units += 2ll * B.n_ct;
    }
    p->max_log_n = std::max(p->max_log_n, ctx->log_n);
  }
  if (smem > smem_optin_limit())
    return fail(ckks_set_error(CKKS_EUNSUPPORTED, "%s: %d B of shared memory per CTA exceed the device's limit", fn,
                               smem));
  p->smem = std::max(smem, 1024);
  p->n_units = n_units;
  int rc = p->max_log_n == 13 ? pb_configure<13>(p, fn) : pb_configure<12>(p, fn);
  if (rc) return fail(rc);

  // ---- counters and device layout
  p->cnt_off.resize(n_buckets);
  size_t n_cnt = 0;
  for (int b = 0; b < n_buckets; ++b) {
    p->cnt_off[b] = n_cnt;
    n_cnt += (size_t)buckets[b].n_ct * (buckets[b].op == CKKS_BATCH_CT_CT ? 3 : 1);
  }
  p->n_cnt = n_cnt;
  const size_t off_ctl = 0;
  const size_t off_cnt = 256;
  p->zero_bytes = align256(off_cnt + n_cnt * sizeof(unsigned));
  const size_t off_slots = p->zero_bytes;
  const size_t off_scr = align256(off_slots + 2 * (size_t)n_units * sizeof(PbSlot));  // both lists
  p->mem_bytes = off_scr + scratch_words * sizeof(u64);
  cudaError_t e = cudaMalloc(&p->mem, p->mem_bytes);
  if (e != cudaSuccess) {
    p->mem = nullptr;
    return fail(ckks_set_error(CKKS_ECUDA, "%s: cudaMalloc(%zu): %s", fn, p->mem_bytes, cudaGetErrorString(e)));
  }
  p->ctl = reinterpret_cast<unsigned*>(p->mem + off_ctl);
  unsigned* cnt = reinterpret_cast<unsigned*>(p->mem + off_cnt);
  p->d_slots = reinterpret_cast<PbSlot*>(p->mem + off_slots);
  u64* scr = reinterpret_cast<u64*>(p->mem + off_scr);
  p->h_buckets.resize(n_buckets);
  for (int b = 0; b < n_buckets; ++b) {
    const ckks_batch_bucket& B = buckets[b];
    const ckks_ctx* ctx = B.ctx;
    PbBucket& D = p->h_buckets[b];
    D.op = B.op;
    D.log_n = ctx->log_n;
    D.level = B.level;
    D.n_ct = B.n_ct;
    D.nq = ctx->n_q;
    D.pt_stride = B.pt_per_ct ? 1 : 0;
    D.a = reinterpret_cast<const u64*>(B.a);
    D.b = reinterpret_cast<const u64*>(B.b);
    D.out = reinterpret_cast<u64*>(B.out);
    D.key = reinterpret_cast<const double*>(B.key);
    D.pi = ctx->d_pi;
    D.tw = ctx->d_tw;
    D.pinv = ctx->d_pinv;
    D.qtinv = ctx->d_qtinv;
    D.cnt = cnt + p->cnt_off[b];
    D.S = CmScratch{};
    if (B.op == CKKS_BATCH_CT_CT) {
      const size_t n = B.n_ct, LN = (size_t)B.level * ctx->n;
      D.S.d01 = scr;
      D.S.d2n = D.S.d01 + n * 2 * LN;
      D.S.d2c = D.S.d2n + n * LN;
      D.S.acc = D.S.d2c + n * LN;
      D.S.accp = D.S.acc + n * 2 * LN;
      scr = D.S.accp + n * 2 * ctx->n;
    }
  }

  std::vector<int> ops(n_buckets), cts(n_buckets), lvls(n_buckets), logs(n_buckets);
  std::vector<double> costs(n_buckets);
  for (int b = 0; b < n_buckets; ++b) {
    ops[b] = buckets[b].op;
    cts[b] = buckets[b].n_ct;
    lvls[b] = buckets[b].level;
    logs[b] = buckets[b].ctx->log_n;
    costs[b] = (double)buckets[b].ctx->n * (2 * buckets[b].level + 3);
  }
  // paired list (a wave: every CTA on one slot, two units each at N = 2^12)
  std::vector<PbJob> jobs((size_t)n_units);
  pb_schedule(n_buckets, ops.data(), cts.data(), lvls.data(), costs.data(),
              (long long)p->grid * 2 * lag_percent / 100, jobs.data());
  std::vector<PbSlot> slots(2 * (size_t)n_units);
  p->n_slots = pb_slots(jobs.data(), n_units, logs.data(), slots.data());
  // phased list, stored after it (a wave: one N = 2^13 unit per CTA, then
  // one N = 2^12 unit per half)
  p->n_whole = pb_phased(n_buckets, ops.data(), cts.data(), lvls.data(), logs.data(), costs.data(),
                         (long long)p->grid * lag_percent / 100, (long long)p->grid * 2 * lag_percent / 100,
                         slots.data() + p->n_slots, &p->n_half);
  p->table = new PbTable();
  for (int b = 0; b < n_buckets; ++b) p->table->b[b] = p->h_buckets[b];
  const long long n_all = p->n_slots + p->n_whole + p->n_half;
  if (n_all)
    e = cudaMemcpy(p->d_slots, slots.data(), (size_t)n_all * sizeof(PbSlot), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e)));
  *out = p;
  return CKKS_OK;
}

extern "C" int ckks_batch_plan_run(ckks_batch_plan* p, long long wait_cycles, int flags, void* stream) {
  const char* fn = "ckks_batch_plan_run";
  CKKS_REQUIRE(p != nullptr, "%s: plan is NULL", fn);
  CKKS_REQUIRE((flags & ~(CKKS_BATCH_RUN_UNMET_WAIT | CKKS_BATCH_RUN_PHASED)) == 0, "%s: unknown flags 0x%x", fn,
               flags);
  int dev = 0;
  cudaGetDevice(&dev);
  CKKS_REQUIRE(dev == p->device, "%s: plan of device %d, current device %d", fn, p->device, dev);
  cudaStream_t st = as_stream(stream);
  cudaError_t e = cudaMemsetAsync(p->mem, 0, p->zero_bytes, st);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  if (p->n_units == 0) return CKKS_OK;
  int unmet = -1;
  if (flags & CKKS_BATCH_RUN_UNMET_WAIT) {
    for (int b = 0; b < p->n_buckets && unmet < 0; ++b)
      if (p->h_buckets[b].op == CKKS_BATCH_CT_CT && p->h_buckets[b].n_ct > 0) unmet = b;
    CKKS_REQUIRE(unmet >= 0, "%s: CKKS_BATCH_RUN_UNMET_WAIT needs a ct x ct item", fn);
  }
  const long long limit = wait_cycles > 0 ? wait_cycles : 2147483647ll;
  ProfSpan span(CKKS_STAGE_BATCH, st);
  const bool paired = (flags & CKKS_BATCH_RUN_PHASED) == 0;
  return p->max_log_n == 13 ? pb_launch<13>(p, paired, limit, unmet, st) : pb_launch<12>(p, paired, limit, unmet, st);
}

extern "C" int ckks_batch_plan_incomplete(ckks_batch_plan* p, int* n_incomplete, uint8_t* bucket_complete) {
  const char* fn = "ckks_batch_plan_incomplete";
  CKKS_REQUIRE(p != nullptr && n_incomplete != nullptr, "%s: NULL pointer argument", fn);
  p->h_cnt.resize(p->n_cnt);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess && p->n_cnt)
    e = cudaMemcpy(p->h_cnt.data(), p->mem + 256, p->n_cnt * sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return ckks_set_error(CKKS_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
  int bad = 0;
  for (int b = 0; b < p->n_buckets; ++b) {
    const PbBucket& B = p->h_buckets[b];
    const unsigned* fin = p->h_cnt.data() + p->cnt_off[b] + (B.op == CKKS_BATCH_CT_CT ? 2 * (size_t)B.n_ct : 0);
    int bad_b = 0;
    for (int i = 0; i < B.n_ct; ++i) bad_b += fin[i] != 2u;
    if (bucket_complete) bucket_complete[b] = bad_b == 0;
    bad += bad_b;
  }
  *n_incomplete = bad;
  return CKKS_OK;
}

extern "C" int ckks_batch_plan_info(const ckks_batch_plan* p, long long* n_units, long long* n_slots, int* grid,
                                    int* smem_bytes, size_t* device_bytes) {
  CKKS_REQUIRE(p != nullptr, "ckks_batch_plan_info: plan is NULL");
  if (n_units) *n_units = p->n_units;
  if (n_slots) *n_slots = p->n_slots;  // the default (paired) list
  if (grid) *grid = p->grid;
  if (smem_bytes) *smem_bytes = p->smem;
  if (device_bytes) *device_bytes = p->mem_bytes;
  return CKKS_OK;
}

extern "C" void ckks_batch_plan_destroy(ckks_batch_plan* p) {
  if (!p) return;
  if (p->mem) cudaFree(p->mem);
  delete p->table;
  delete p;
}
