// Device-side building blocks shared by every kernel of the delayed-pivoting
// LU: index helpers, the per-factorisation state block that keeps all pivot
// decisions on the device, and bounded spin waits.
#pragma once

#include <cstddef>
#include <atomic>
#include <map>
#include <mutex>
#include <utility>
#include <cstdint>
#include <cuda_runtime.h>

namespace dp {

// Kernel launches issued by this library since it was loaded (every launch
// site calls note_launch); read through dp_kernel_launches().
inline std::atomic<long long> g_kernel_launches{0};
inline void note_launch(long long k = 1) {
  g_kernel_launches.fetch_add(k, std::memory_order_relaxed);
}

// Raises the dynamic shared-memory limit of kernel `func` on the current
// device to at least `bytes`, calling the runtime only when the limit grows
// (the call costs milliseconds for large limits, far more than a launch).
inline bool ensure_smem(const void* func, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lock(m);
  size_t& have = done[{func, dev}];
  if (have >= bytes) return true;
  if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
      cudaSuccess)
    return false;
  have = bytes;
  return true;
}

// Resident CTAs per SM of `func` at `threads` x `smem` on the current device,
// computed once per (kernel, device, smem); 0 on error.
inline int occupancy_once(const void* func, int threads, size_t smem) {
  static std::mutex m;
  static std::map<std::pair<std::pair<const void*, int>, size_t>, int> memo;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(m);
  auto key = std::make_pair(std::make_pair(func, dev), smem);
  auto it = memo.find(key);
  if (it != memo.end()) return it->second;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem) != cudaSuccess)
    per_sm = 0;
  memo[key] = per_sm;
  return per_sm;
}

// Multiprocessors of the current device (memoised per device).
inline int sm_count() {
  static std::mutex m;
  static std::map<int, int> memo;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(m);
  auto it = memo.find(dev);
  if (it != memo.end()) return it->second;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 0;
  memo[dev] = sms;
  return sms;
}

// Status codes shared by kernels and host (values of the C ABI).
enum : int {
  kOk = 0,
  kInvalidArgument = 1,
  kAllocationFailed = 2,
  kCudaFailure = 3,
  kLibraryFailure = 4,  // reference name: cublas_failure
  kDeviceTimeout = 5,   // a bounded device wait gave up
};

__host__ __device__ inline size_t idx(long long row, long long col, long long ld) {
  return static_cast<size_t>(row) + static_cast<size_t>(col) * static_cast<size_t>(ld);
}

// One pivot candidate of the full (2-D) search.  Ordering follows the
// reference (delayed_lu_cuda/delayed_dgetrf_cuda.cu:13-20): larger magnitude
// wins; equal magnitudes go to the earlier element in column-major order
// (smaller column, then smaller row); NaN never wins.
struct Cand {
  double val;
  int row;
  int col;
  double sec;  // runner-up: the largest other magnitude seen (near-tie detector)
};

__device__ __forceinline__ bool cand_better(const Cand& a, const Cand& b) {
  // true iff a beats b
  if (a.val > b.val) return true;
  if (a.val == b.val) {
    if (a.col != b.col) return a.col < b.col;
    return a.row < b.row;
  }
  return false;
}

// Merges two candidates over disjoint element sets (winner by cand_better,
// runner-up the largest magnitude that did not win; NaN is never taken).
__device__ __forceinline__ Cand cand_merge(const Cand& a, const Cand& b) {
  Cand r = cand_better(b, a) ? b : a;
  const Cand& lose = cand_better(b, a) ? a : b;
  r.sec = fmax(r.sec, fmax(lose.val, lose.sec));
  return r;
}

// Device-resident state of one factorisation.  Written by kernels, read by
// the host once per panel (a few bytes) or once per fallback.
struct State {
  int status;      // kOk or an error code (e.g. kDeviceTimeout)
  int stop_k;      // panel stopped at this step (no acceptable column pivot), -1 if not
  int swap_count;  // number of (dst, src) pairs below the panel in the swap list
  int block_changed;  // block rows [begin, end) whose content changed in the last panel
  Cand fallback;   // result of the last 2-D / column-fallback search
  unsigned int search_done;  // last-block-done counter of the search kernels
  unsigned int barrier_exit; // exit counter of the panel kernel
  int pad1[2];
  // Near-tie detector: every pivot decision (column search of a panel step,
  // fallback search) also reduces the runner-up magnitude; a decision whose
  // winner beats the runner-up by at most kNearTieC (k + 1) u |winner| (u =
  // 2^-53, k the step) could change under another summation order and is
  // counted as order-sensitive.  Decisions on a zero winner (delay / stop)
  // are exact and never count.
  unsigned long long ties_checked;  // decisions whose runner-up was compared
  unsigned long long near_ties;     // order-sensitive decisions among them
  unsigned long long closeness;     // bits of max(second / best) over the checked decisions
};

constexpr double kNearTieC = 4.0;

// Records one pivot decision of step k with winner magnitude `best` and
// runner-up `second` (both >= 0; NaN never reaches here).  Called by one
// thread per decision, inside the panels' per-column critical path: only
// reduction atomics whose results are unused, so the thread issues them and
// goes on without waiting for a round trip to memory.
__device__ __forceinline__ void note_decision(State* st, long long k, double best, double second) {
  atomicAdd(&st->ties_checked, 1ull);
  if (best > 0.0) {
    if (best - second <= kNearTieC * (double)(k + 1) * 0x1p-53 * best)
      atomicAdd(&st->near_ties, 1ull);
    atomicMax(&st->closeness, (unsigned long long)__double_as_longlong(second / best));
  }
}

// The same record kept in registers by the one thread of a panel kernel that
// records its decisions, and flushed to the state once, when it finishes:
// the per-column critical path then carries no memory operation for it.
// The largest ratio second / best is kept as its (second, best) pair,
// compared by cross products, so that the one division happens at the flush.
struct DecisionTally {
  unsigned long long checked = 0, near = 0;
  double c_sec = 0.0, c_best = 1.0;  // pair of the largest ratio so far
  __device__ __forceinline__ void note(long long k, double best, double second) {
    ++checked;
    if (best > 0.0) {
      if (best - second <= kNearTieC * (double)(k + 1) * 0x1p-53 * best) ++near;
      if (second * c_best > c_sec * best) {
        c_sec = second;
        c_best = best;
      }
    }
  }
  __device__ __forceinline__ void flush(State* st) const {
    if (checked) atomicAdd(&st->ties_checked, checked);
    if (near) atomicAdd(&st->near_ties, near);
    if (c_sec > 0.0)
      atomicMax(&st->closeness, (unsigned long long)__double_as_longlong(c_sec / c_best));
  }
};

// Bounded wait: every spin in this library gives up after kSpinLimitNs of
// wall time, records kDeviceTimeout in the state and lets the caller return.
constexpr unsigned long long kSpinLimitNs = 4000000000ull;  // 4 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.volatile.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// 16-byte volatile vector access: both words of a tagged candidate travel in
// one request (each word carries its own tag, so a torn read is detected).
// GPU-scope relaxed accesses (system-scope volatile would also order against
// the host and peers, which these device-local flags do not need).
__device__ __forceinline__ void ld_volatile_v2u64(const unsigned long long* p,
                                                  unsigned long long& a, unsigned long long& b) {
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ void st_volatile_v2u64(unsigned long long* p, unsigned long long a,
                                                  unsigned long long b) {
  asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}

// Release / acquire fence at GPU scope (cumulative: orders this thread's
// earlier writes, and those it has observed, before its later writes).
__device__ __forceinline__ void fence_acq_rel_gpu() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

__device__ __forceinline__ int ld_volatile_i32(const int* p) {
  int v;
  asm volatile("ld.volatile.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

}  // namespace dp
