// Optional per-kernel-family device timing shared by the library's drivers
// (dp_stats_enable / _get / _reset / _families in getrf.cu).
#pragma once
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "delayed_pivoting_b200.h"

namespace dp {

// Optional per-kernel-family device timing (dp_stats_enable): CUDA events
// around each launch group on the launching stream, read after the call's
// final synchronisation, plus the algorithmic flops / bytes of each group.
inline std::mutex g_stats_mutex;
inline dp_kernel_stats g_stats;
inline bool g_stats_on = false;
inline unsigned g_stats_mask = ~0u;  // kernel families recorded while enabled

// Events are recycled across calls (creating them per launch costs more
// host time than the launches themselves).  Guarded by g_stats_mutex.
inline std::vector<cudaEvent_t> g_event_pool;
inline std::mutex g_pool_mutex;

inline cudaEvent_t event_get() {
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

inline void event_put(cudaEvent_t e) {
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  g_event_pool.push_back(e);
}

// Timeline dump (environment variable DP_TIMELINE=<file>, with dp_stats
// enabled): every recorded launch group is appended to the file as
// "call lane family start_ms end_ms launches", times relative to an event
// recorded on the caller's stream when the call starts; lane 0 is the
// critical-path stream, lane 1 the trailing-update stream.
inline const char* timeline_path() {
  static const char* p = std::getenv("DP_TIMELINE");
  return p && p[0] ? p : nullptr;
}
inline long long g_timeline_calls = 0;

struct Recorder {
  struct Mark {
    int fam;
    cudaEvent_t e0, e1;
    double flops, bytes;
    int launches;
  };
  bool on = false;
  unsigned mask = ~0u;
  cudaStream_t st = nullptr;
  std::vector<Mark> marks;
  int cur = -1;
  int lane = 0;
  cudaEvent_t base = nullptr;  // timeline origin (nullptr: no timeline)
  explicit Recorder(cudaStream_t s) : st(s) {
    std::lock_guard<std::mutex> lock(g_stats_mutex);
    on = g_stats_on;
    mask = g_stats_mask;
  }
  void begin(int fam) {
    cur = -1;
    if (!on || !(mask >> fam & 1u)) return;
    Mark mk{fam, nullptr, nullptr, 0.0, 0.0, 0};
    mk.e0 = event_get();
    mk.e1 = event_get();
    cudaEventRecord(mk.e0, st);
    marks.push_back(mk);
    cur = (int)marks.size() - 1;
  }
  void end(double flops, double bytes, int launches) {
    if (!on || cur < 0) return;
    Mark& mk = marks[cur];
    cudaEventRecord(mk.e1, st);
    mk.flops = flops;
    mk.bytes = bytes;
    mk.launches = launches;
    cur = -1;
  }
  // Called after the stream has been synchronised.
  void flush(bool ok) {
    if (!on) return;
    std::lock_guard<std::mutex> lock(g_stats_mutex);
    FILE* tl = ok && base && timeline_path() ? std::fopen(timeline_path(), "a") : nullptr;
    for (Mark& mk : marks) {
      float t0 = 0.f, t1 = 0.f;
      if (tl && mk.e1 && cudaEventElapsedTime(&t0, base, mk.e0) == cudaSuccess &&
          cudaEventElapsedTime(&t1, base, mk.e1) == cudaSuccess)
        std::fprintf(tl, "%lld %d %d %.4f %.4f %d\n", g_timeline_calls, lane, mk.fam, t0, t1,
                     mk.launches);
      float ms = 0.f;
      if (ok && mk.e1 && cudaEventElapsedTime(&ms, mk.e0, mk.e1) == cudaSuccess) {
        g_stats.ms[mk.fam] += ms;
        g_stats.flops[mk.fam] += mk.flops;
        g_stats.bytes[mk.fam] += mk.bytes;
        g_stats.launches[mk.fam] += mk.launches;
      }
      event_put(mk.e0);
      event_put(mk.e1);
    }
    if (ok) g_stats.calls += 1;
    if (tl) std::fclose(tl);
    marks.clear();
  }
};

}  // namespace dp
