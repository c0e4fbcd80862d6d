// Host driver of the delayed-pivoting LU and the library's entry points
// (C++ drop-in symbols of delayed_lu_cuda/delayed_dgetrf_cuda.hpp and the
// extern "C" ABI of include/delayed_pivoting_b200.h).
//
// Control flow follows delayed_lu/delayed_dgetrf.cpp:129-251 and its GPU twin
// delayed_lu_cuda/delayed_dgetrf_cuda.cu:251-368, with the per-pivot work moved
// to the device: one cooperative panel launch factors a whole panel (all
// column searches, acceptance tests, swaps, scalings and rank-1 updates stay
// on the GPU) and the host reads a 64-byte state block once per panel, where
// the reference made 2 launches + a D2H copy + a stream sync per column.
//   normal panel  : laswp (rows outside the panel) -> TRSM (U12) -> GEMM (A22)
//   panel stopped at k (no acceptable column pivot, dgetrf.cpp:182-218):
//                   laswp of the executed steps -> materialize far columns
//                   (TRSM + GEMM of width k - begin) -> full or column
//                   fallback search -> delay (info = k) or swap row/column and
//                   restart the panel at k with the pivot in place.
// With look-ahead (the default for more than one outer block) the trailing
// update of a finished outer block is split: the next block's columns are
// updated on a high-priority stream that then factors that block's panels,
// while the rest of the update runs on a low-priority stream behind them.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <vector>

#include "delayed_dgetrf_cuda.hpp"
#include "delayed_pivoting_b200.h"
#include "dp_stats.h"
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int kDefaultNb = 64;
constexpr int kDefaultNbOuter = 256;
constexpr int kMaxPanelWidth = 128;   // TRSM stages L11 (w x w) in shared memory
constexpr int kDefaultPanelRows = 256;
constexpr int kMaxSearchBlocks = 1024;

struct DeviceInfo {
  int sms = 0;
  int smem_optin = 0;
  int max_cluster = 0;  // largest cluster the cluster panel kernel may use (0: none)
  bool ready = false;
};

std::mutex g_dev_mutex;
DeviceInfo g_dev[64];

int device_info(DeviceInfo& out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return kCudaFailure;
  std::lock_guard<std::mutex> lock(g_dev_mutex);
  DeviceInfo& d = g_dev[dev];
  if (!d.ready) {
    if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
            cudaSuccess)
      return kCudaFailure;
    if (cudaFuncSetAttribute(panel_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             d.smem_optin - 1024) != cudaSuccess)
      return kCudaFailure;
    d.max_cluster = 0;
    // the register-sub-panel cluster kernels, one instance per rows-per-thread
    for (int r = 256; r <= panel_reg_max_rows(); r *= 2) {
      const void* f = panel_reg_kernel_for(r);
      if (!f || cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     d.smem_optin - 1024) != cudaSuccess ||
          cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
              cudaSuccess)
        return kCudaFailure;
    }
    if (cudaFuncSetAttribute(panel_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             d.smem_optin - 1024) == cudaSuccess) {
      cudaFuncSetAttribute(panel_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      for (int c : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(panel_cluster_threads());
        cfg.dynamicSmemBytes = (size_t)d.smem_optin - 1024;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, panel_cluster_kernel, &cfg) == cudaSuccess &&
            clusters >= 1) {
          d.max_cluster = c;
          break;
        }
      }
      cudaGetLastError();
    }
    d.ready = true;
  }
  out = d;
  return kOk;
}

struct Options {
  int precision = DP_PRECISION_FP64;
  int panel_kernel = 0;  // 0 automatic, 1 cluster, 2 multi-CTA grid, 3 shared-memory cluster
  int nb = kDefaultNb;
  int nb_outer = kDefaultNbOuter;
  double threshold = 0.0;
  int policy = DP_POLICY_FULL_PIVOT;
  int panel_rows = kDefaultPanelRows;
  int lookahead = 0;  // 0 automatic (more than one outer block), 1 on, 2 off
};

struct Workspace {
  char* base = nullptr;
  size_t bytes = 0;
  State* state = nullptr;
  int* d_ipiv = nullptr;
  int* d_jpiv = nullptr;
  unsigned long long* slots = nullptr;
  double* xdata = nullptr;
  double* rowk = nullptr;
  int* swap_block = nullptr;
  int* swap_extra = nullptr;
  Cand* cands = nullptr;
  void* mixed = nullptr;   // BF16 operand scratch of the tensor-core update (mixed precision)
  void* mixed1 = nullptr;  // the same for the next outer block's update on the panel stream
  // Look-ahead: swap lists of the panels of an outer block, kept until the
  // block completes (two buffers, alternating between consecutive blocks;
  // panel [b, e) of block [B, E) at defer_blk + (b - B), defer_ext + 2 (b - B)),
  // and the error word of the kernels on the trailing-update stream.
  int* defer_blk = nullptr;
  int* defer_ext = nullptr;
  int defer_cap = 0;
  int* aux_status = nullptr;
  // Block solves of the outer blocks as GEMMs: T = I - L11^{-1} of an outer
  // block (two, alternating between consecutive blocks like the deferred swap
  // lists; tinv_ld x tinv_ld each) and copies of the block rows being solved
  // (tcopy1: the panel stream's, up to copy1_cols columns; tcopy2: the
  // trailing stream's or the only stream's, up to copy2_cols columns).
  // Absent (tinv == nullptr) in the allocation-free workspace.
  double* tinv = nullptr;
  double* tcopy1 = nullptr;
  double* tcopy2 = nullptr;
  int tinv_ld = 0;
  char* scratch = nullptr;  // from here on, every region is written before it is read
  int max_ctas = 0;
  int w_max = 0;
};

// dp_block_solve: 0 automatic (inverse), 1 inverse, 2 substitution.
std::atomic<int> g_block_solve{0};

// Geometry of the block solves by inverse (Workspace::tinv).
struct InvPlan {
  int ld = 0;              // 0: no block solves by inverse
  long long copy1_cols = 0, copy2_cols = 0;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Lays the workspace out from `base` (nullptr: only computes the size).
size_t layout_workspace(Workspace& ws, char* base, int pivots, int max_ctas, int w_max,
                        size_t mixed_bytes, int defer_cap = 0, size_t mixed1_bytes = 0,
                        const InvPlan& inv = InvPlan{}) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align_up(off + bytes, 256);
    return base ? base + at : nullptr;
  };
  ws.max_ctas = max_ctas;
  ws.w_max = w_max;
  ws.state = reinterpret_cast<State*>(take(sizeof(State)));
  ws.d_ipiv = reinterpret_cast<int*>(take(sizeof(int) * (size_t)std::max(pivots, 1)));
  ws.d_jpiv = reinterpret_cast<int*>(take(sizeof(int) * (size_t)std::max(pivots, 1)));
  ws.slots = reinterpret_cast<unsigned long long*>(
      take(sizeof(unsigned long long) * 2 * 4 * (size_t)max_ctas * max_ctas * 2));
  ws.xdata = reinterpret_cast<double*>(take(sizeof(double) * 4 * (size_t)max_ctas * (w_max + 1)));
  ws.rowk = reinterpret_cast<double*>(take(sizeof(double) * 4 * (size_t)(w_max + 1)));
  ws.swap_block = reinterpret_cast<int*>(take(sizeof(int) * (size_t)w_max));
  ws.swap_extra = reinterpret_cast<int*>(take(sizeof(int) * 2 * (size_t)w_max));
  ws.cands = reinterpret_cast<Cand*>(take(sizeof(Cand) * kMaxSearchBlocks));
  ws.defer_cap = defer_cap;
  if (defer_cap > 0) {
    ws.defer_blk = reinterpret_cast<int*>(take(sizeof(int) * 2 * (size_t)defer_cap));
    ws.defer_ext = reinterpret_cast<int*>(take(sizeof(int) * 4 * (size_t)defer_cap));
    ws.aux_status = reinterpret_cast<int*>(take(sizeof(int)));
  }
  ws.scratch = base ? base + off : nullptr;
  ws.mixed = mixed_bytes ? reinterpret_cast<void*>(take(mixed_bytes)) : nullptr;
  ws.mixed1 = mixed1_bytes ? reinterpret_cast<void*>(take(mixed1_bytes)) : nullptr;
  ws.tinv_ld = inv.ld;
  if (inv.ld > 0) {
    const size_t ld = (size_t)inv.ld;
    ws.tinv = reinterpret_cast<double*>(take(sizeof(double) * 2 * ld * ld));
    ws.tcopy1 = inv.copy1_cols > 0
                    ? reinterpret_cast<double*>(take(sizeof(double) * ld * (size_t)inv.copy1_cols))
                    : nullptr;
    ws.tcopy2 = reinterpret_cast<double*>(take(sizeof(double) * ld * (size_t)inv.copy2_cols));
  }
  ws.base = base;
  ws.bytes = off;
  return off;
}

// Picks the panel kernel's CTA count G and rows per CTA R so that the R x w
// slice fits in shared memory; narrows the panel when it cannot fit.
bool plan_panel(int rows, int& w, int target_rows, const DeviceInfo& di, int& G, int& R) {
  const size_t budget = (size_t)di.smem_optin - 1024;
  while (w >= 1) {
    // pivot / old-row buffers, one padding row of the odd column stride, slack
    const size_t fixed = 2 * (size_t)(w + 1) * sizeof(double) + (size_t)w * sizeof(double) + 64;
    const long long max_r = (long long)((budget - fixed) / ((size_t)w * sizeof(double) + sizeof(int)));
    long long g = (rows + (long long)target_rows - 1) / target_rows;
    g = std::max(1LL, std::min<long long>(g, di.sms));
    long long r = (rows + g - 1) / g;
    if (r > max_r) {
      g = std::min<long long>(di.sms, (rows + max_r - 1) / max_r);
      r = (rows + g - 1) / g;
    }
    if (r <= max_r) {
      G = (int)((rows + r - 1) / r);  // every CTA owns at least one row
      R = (int)r;
      return true;
    }
    w /= 2;
  }
  return false;
}

// Cluster panel: C CTAs (one cluster) of R rows each, about target_rows per
// CTA (fewer CTAs per panel: less SM time per column, more latency); the
// R x w slice per CTA must fit in shared memory.  Returns false when even an
// 8-wide panel does not fit (very tall panels then use panel_factor_kernel).
// `reg` selects the kernel: the register-sub-panel one where R allows it
// (unless `smem_only`), else the shared-memory one.
bool plan_cluster(int rows, int& w, const DeviceInfo& di, int& C, int& R,
                  int target_rows = kDefaultPanelRows, bool* reg = nullptr,
                  bool smem_only = false) {
  if (di.max_cluster <= 0) return false;
  const size_t budget = (size_t)di.smem_optin - 1024 - 512;
  const long long t = std::max(1, target_rows);
  C = (int)std::min<long long>(di.max_cluster, std::max(1LL, ((long long)rows + t - 1) / t));
  R = (rows + C - 1) / C;
  const bool use_reg = !smem_only && R <= panel_reg_max_rows();
  if (reg) *reg = use_reg;
  auto bytes = [&](int ww) {
    return use_reg ? panel_reg_smem_bytes(ww, R) : panel_cluster_smem_bytes(ww, R);
  };
  int wf = w;
  while (wf >= 1 && bytes(wf) > budget) --wf;
  if (wf < std::min(w, 8)) return false;
  if (wf < w) w = wf >= 16 ? (wf & ~7) : wf;
  return true;
}

// Near-tie report of the calling thread's last factorisation (every entry
// point is synchronous, so "last" is well defined per host thread).
thread_local dp_getrf_report g_report = {0, 0, 0.0, -1, {0, 0, 0}};

void set_report(const State& s, int info) {
  g_report.decisions = (long long)s.ties_checked;
  g_report.near_ties = (long long)s.near_ties;
  double c = 0.0;
  std::memcpy(&c, &s.closeness, sizeof(c));
  g_report.max_closeness = c;
  g_report.info = info;
}

void clear_report() { g_report = dp_getrf_report{0, 0, 0.0, -1, {0, 0, 0}}; }

#define DP_CHECK_CUDA(call)                       \
  do {                                            \
    if ((call) != cudaSuccess) return kCudaFailure; \
  } while (0)

// Host-side phase trace (environment variable DP_TRACE=1): accumulated wall
// time spent waiting in read_state versus issuing work, printed per call.
struct HostTrace {
  bool on = false;
  double wait_s = 0.0, total_s = 0.0;
  long long waits = 0;
  std::chrono::steady_clock::time_point t0;
  HostTrace() {
    const char* e = std::getenv("DP_TRACE");
    on = e && e[0] == '1';
    t0 = std::chrono::steady_clock::now();
  }
  ~HostTrace() {
    if (!on) return;
    total_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::fprintf(stderr, "[dp trace] call %.3f ms, %lld state reads waited %.3f ms\n",
                 total_s * 1e3, waits, wait_s * 1e3);
  }
};
thread_local HostTrace* g_trace = nullptr;

int read_state(State& hs, const Workspace& ws, cudaStream_t st) {
  const auto t = std::chrono::steady_clock::now();
  DP_CHECK_CUDA(cudaMemcpyAsync(&hs, ws.state, sizeof(State), cudaMemcpyDeviceToHost, st));
  DP_CHECK_CUDA(cudaStreamSynchronize(st));
  if (g_trace && g_trace->on) {
    g_trace->wait_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
    g_trace->waits += 1;
  }
  return kOk;
}

// Per-kernel-family device timing: struct Recorder in dp_stats.h.

double panel_flops(int m, int begin, int w) {
  double f = 0.0;
  for (int s = 0; s < w; ++s) {
    const double below = (double)m - begin - s - 1;
    if (below > 0) f += below * (2.0 * (w - s - 1) + 1.0);
  }
  return f;
}

// Blocked forward substitution U <- L^{-1} A for rows [r0, r0 + W) and
// columns [c0, c0 + nc), L unit lower at a(r0, r0); diagonal blocks of at
// most trsm_max_width() are solved by the TRSM kernel, the blocks below them
// by the GEMM kernel.
void trsm_blocked(double* a, long long lda, int r0, int W, int c0, int nc, cudaStream_t st,
                  Recorder& rec, const int* gate = nullptr) {
  if (W <= 1 || nc <= 0) return;
  const int tw = trsm_max_width();
  for (int b = 0; b < W; b += tw) {
    const int wb = std::min(tw, W - b);
    if (wb > 1) {
      rec.begin(DP_KFAM_TRSM);
      launch_trsm_unit_lower(a, lda, r0 + b, wb, c0, nc, st, gate);
      rec.end((double)wb * (wb - 1) * nc, 8.0 * (0.5 * wb * wb + 2.0 * wb * nc), 1);
    }
    const int rows_below = W - b - wb;
    if (rows_below > 0) {
      rec.begin(DP_KFAM_GEMM);
      launch_gemm_minus(rows_below, nc, wb, a + idx(r0 + b + wb, r0 + b, lda), lda,
                        a + idx(r0 + b, c0, lda), lda, a + idx(r0 + b + wb, c0, lda), lda, st,
                        gate);
      rec.end(2.0 * rows_below * (double)nc * wb,
              8.0 * ((double)rows_below * wb + (double)wb * nc + 2.0 * rows_below * (double)nc), 1);
    }
  }
}

// Brings columns [c0, n_end) up to date with the eliminated steps
// [s0, s0 + W): blocked TRSM on rows [s0, s0 + W), then
// A(r_gemm:m, c0:n_end) -= L(r_gemm:m, s0:s0+W) * U(s0:s0+W, c0:n_end).
// When `mixed_ws` is set the rank-W update runs on the tensor cores (BF16
// split into `terms` pieces, FP32 accumulation); the TRSM always runs in FP64.
// A non-null `gate` (FP64 only) makes the kernels do nothing once *gate >= 0.
// A non-null `bi` holding T = I - L^{-1} of the W x W block at a(s0, s0)
// solves blocks wider than trsm_max_width() as U = B - T C, C a copy of B
// (one copy and one GEMM instead of the chain of 64-row solves and updates).
struct BlockInv {
  const double* T = nullptr;
  long long ldt = 0;
  double* copy = nullptr;  // ldt x (columns) doubles
};

// `solved`: the block rows already hold U12 (the panel's laswp solved them).
int update_columns(double* a, long long lda, int m, int s0, int W, int r_gemm, int c0, int n_end,
                   cudaStream_t st, Recorder& rec, void* mixed_ws = nullptr,
                   int* status = nullptr, int terms = 2, const int* gate = nullptr,
                   const BlockInv* bi = nullptr, bool solved = false) {
  const int nc = n_end - c0;
  if (W <= 0 || nc <= 0) return kOk;
  if (solved) {
    // U12 in place
  } else if (bi && bi->T && W > trsm_max_width() && W <= bi->ldt) {
    rec.begin(DP_KFAM_TRSM);
    launch_copy_block(a + idx(s0, c0, lda), lda, bi->copy, W, W, nc, st);
    launch_gemm_minus(W, nc, W, bi->T, bi->ldt, bi->copy, W, a + idx(s0, c0, lda), lda, st, gate);
    rec.end(2.0 * W * (double)W * nc, 8.0 * ((double)W * W + 4.0 * W * (double)nc), 2);
  } else {
    trsm_blocked(a, lda, s0, W, c0, nc, st, rec, gate);
  }
  const int M = m - r_gemm;
  if (M <= 0) return kOk;
  const double fl = 2.0 * M * (double)nc * W;
  const double by = 8.0 * ((double)M * W + (double)W * nc + 2.0 * M * (double)nc);
  if (mixed_ws) {
    rec.begin(DP_KFAM_GEMM_MIXED);
    const int e = launch_gemm_minus_mixed(M, nc, W, a + idx(r_gemm, s0, lda), lda,
                                          a + idx(s0, c0, lda), lda, a + idx(r_gemm, c0, lda), lda,
                                          mixed_ws, terms, status, st);
    rec.end(fl, by, 3);
    return e;
  }
  rec.begin(DP_KFAM_GEMM);
  launch_gemm_minus(M, nc, W, a + idx(r_gemm, s0, lda), lda, a + idx(s0, c0, lda), lda,
                    a + idx(r_gemm, c0, lda), lda, st, gate);
  rec.end(fl, by, 1);
  return kOk;
}

// Streams and events of the look-ahead schedule, created once per host thread
// and device: `panel` (highest priority) carries the critical path - panels,
// in-block updates, the next outer block's columns - and `trail` (lowest
// priority) the bulk of each trailing update, so that panel CTAs are placed
// ahead of waiting GEMM tiles.
// `left` (lowest priority) carries the row swaps of the finished L columns
// left of each outer block, which nothing reads until the factorisation
// ends, beside the trailing update instead of in front of it.
struct Lanes {
  cudaStream_t panel = nullptr, trail = nullptr, left = nullptr;
  cudaEvent_t fork = nullptr, block = nullptr, next = nullptr, join = nullptr, ldone = nullptr,
              tdone = nullptr;
  bool ready = false;
  bool init() {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&panel, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&trail, cudaStreamNonBlocking, least) != cudaSuccess ||
        cudaStreamCreateWithPriority(&left, cudaStreamNonBlocking, least) != cudaSuccess)
      return false;
    for (cudaEvent_t* e : {&fork, &block, &next, &join, &ldone, &tdone})
      if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return false;
    ready = true;
    return true;
  }
  ~Lanes() {
    for (cudaEvent_t e : {fork, block, next, join, ldone, tdone})
      if (e) cudaEventDestroy(e);
    if (panel) cudaStreamDestroy(panel);
    if (trail) cudaStreamDestroy(trail);
    if (left) cudaStreamDestroy(left);
  }
};
thread_local Lanes g_lanes[64];

Lanes* lanes_for_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  Lanes& l = g_lanes[dev];
  if (!l.ready && !l.init()) {
    cudaGetLastError();
    return nullptr;
  }
  return &l;
}

// Where factorize issues its work: `s1` always; `s2` (look-ahead) takes the
// trailing updates right of the next outer block, ordered against `s1` by
// the events `block` (s1 -> s2: an outer block and the next block's columns
// are done) and `next` (s2 -> s1: the columns of the block after next have
// this block's update).  `s3` takes the swaps of the columns left of each
// block, after `block` and after `tdone` (s2 -> s3: the previous block's
// trailing update, the last reader of its L columns, is done); `ldone`
// (s3 -> s1) marks them applied.
struct Schedule {
  cudaStream_t s1 = nullptr, s2 = nullptr, s3 = nullptr;
  Recorder* r1 = nullptr;
  Recorder* r2 = nullptr;
  Recorder* r3 = nullptr;
  cudaEvent_t block = nullptr, next = nullptr, ldone = nullptr, tdone = nullptr;
};

// Applies the deferred swap lists of the panels [B, B + sum widths) of an
// outer block to the columns [c0, c1) and [c2, c3).
int apply_deferred(double* a, long long lda, const int* blk, const int* ext, int B,
                   const std::vector<int>& widths, int c0, int c1, int c2, int c3,
                   cudaStream_t st, Recorder& rec) {
  const long long cols = (long long)std::max(0, c1 - c0) + std::max(0, c3 - c2);
  if (widths.empty() || cols <= 0) return kOk;
  double moved = 0.0;  // at most: every block row and one row below it per step
  for (int w : widths) moved += 2.0 * w;
  rec.begin(DP_KFAM_LASWP);
  const int launches = launch_laswp_seq(a, lda, blk, ext, B, widths.data(), (int)widths.size(),
                                        c0, c1, c2, c3, st);
  rec.end(0.0, 16.0 * moved * (double)cols, std::max(launches, 0));
  return launches < 0 ? kInvalidArgument : kOk;
}

// Two-level blocked delayed LU.  An outer block [B, E) of width NB is
// factored as a sequence of inner panels [b, e) of width nb (the panel
// kernel); after each inner panel its row swaps are applied to the columns
// outside it and the rest of the outer block [e, E) is updated (rank nb);
// the columns right of the outer block receive one rank-NB update when the
// block completes.  When a panel stops at step k (no acceptable column
// pivot) every column right of the stopped panel is brought up to date for
// the steps [B, k) (delayed_dgetrf.cpp:183-186 materialize), the fallback
// search runs on the true Schur complement A(k:m, k:n), and the factorisation
// either delays from k (info = k) or swaps the chosen pivot to (k, k) and
// restarts a new outer block at k with that pivot positioned
// (delayed_dgetrf.cpp:188-218).  Block sizes only change rounding, never the
// pivot decisions.
//
// Look-ahead (sc.s2 set): inside an outer block a panel's swaps reach only
// the block's own columns; the swaps outside the block are kept (per panel)
// and applied when the block completes.  Then, on s1: the block's swaps and
// update on the next block's columns [E, NE); on s2, behind them: the swaps
// on [0, B) and [NE, n), the update of the block after next [NE, NNE)
// (event `next`), and the update of [NNE, n).  The next block's panels run
// on s1 while s2 works; before touching [NE, NNE) s1 waits for `next`.  A
// stop drains s2 and applies the block's kept swaps everywhere, which
// restores the state of the unscheduled order before the materialize /
// search logic runs.  Every element receives the same operations in the
// same order either way, so the schedule changes no result.
//
// With look-ahead the cluster panels of a block are also enqueued without a
// host round trip each: a panel that stops records stop_k, and every kernel
// enqueued after it (later panels, their swaps, the in-block updates) reads
// the word when it starts and does nothing.  The host reads the state once
// per block, finds the stopped panel from stop_k, and proceeds exactly as if
// it had stopped there.  (The grid-wide cooperative panel keeps a round trip
// per panel, with s2 drained before it.)
int factorize(int m, int n, double* a, long long lda, const Options& o, Workspace& ws,
              const DeviceInfo& di, const Schedule& sc, int& info) {
  cudaStream_t st = sc.s1;
  Recorder& rec = *sc.r1;
  const bool la = sc.s2 != nullptr;
  const int pivots = std::min(m, n);
  rec.begin(DP_KFAM_OTHER);
  launch_identity_records(ws.d_ipiv, ws.d_jpiv, pivots, st);
  rec.end(0.0, 8.0 * pivots, 1);
  DP_CHECK_CUDA(cudaGetLastError());
  info = pivots;
  int B = 0, parity = 0, half = 0;
  bool positioned = false, pending = false;
  State hs;
  const int NB = std::max(o.nb_outer, o.nb);
  const int terms = mixed_terms(o.precision);
  void* mixed_ws = terms ? ws.mixed : nullptr;
  int* const stop_word = &ws.state->stop_k;
  std::vector<int> widths;  // the current block's panels (look-ahead)
  if (la) DP_CHECK_CUDA(cudaMemsetAsync(stop_word, 0xFF, sizeof(int), st));  // stop_k = -1
  // T = I - L^{-1} of the W x W block at a(s0, s0) into buffer `which`, when
  // the block is solved by inverse (wider than the TRSM kernel's blocks);
  // returns the solve's operands for the panel stream and the other stream
  auto block_inverse = [&](int s0, int W, int which, BlockInv& on1, BlockInv& on2) {
    on1 = on2 = BlockInv{};
    if (!ws.tinv || W <= trsm_max_width() || W > ws.tinv_ld) return;
    double* T = ws.tinv + (size_t)which * ws.tinv_ld * ws.tinv_ld;
    rec.begin(DP_KFAM_TRSM);
    launch_lower_inverse(a + idx(s0, s0, lda), lda, W, T, ws.tinv_ld, st);
    rec.end((double)W * W * W / 3.0, 8.0 * (0.5 * (double)W * W + (double)W * W), 1);
    on1 = BlockInv{T, ws.tinv_ld, ws.tcopy1 ? ws.tcopy1 : ws.tcopy2};
    on2 = BlockInv{T, ws.tinv_ld, ws.tcopy2};
  };
  BlockInv inv1, inv2;
  while (B < pivots) {
    const int E = std::min(pivots, B + NB);
    int* blk = la ? ws.defer_blk + (size_t)half * ws.defer_cap : ws.swap_block;
    int* ext = la ? ws.defer_ext + (size_t)2 * half * ws.defer_cap : ws.swap_extra;
    // extra pairs are written from the front of each panel's region: the
    // rest must read as "no pair" (destination -1)
    if (la) DP_CHECK_CUDA(cudaMemsetAsync(ext, 0xFF, sizeof(int) * 2 * (size_t)(E - B), st));
    widths.clear();
    int b = B, e = B, stop = -1;
    bool unread = false;  // enqueued panels whose state the host has not read
    while (b < E) {
      int w = std::min(std::min(o.nb, ws.w_max), E - b);
      int G = 1, R = 1;
      // short panels: one CTA, rows in registers (automatic choice only)
      const bool use_small = o.panel_kernel == 0 && m - b <= panel_small_max_rows();
      if (use_small) w = std::min(w, panel_small_max_width());
      bool use_reg = false;
      const bool use_cluster =
          !use_small && o.panel_kernel != 2 &&
          plan_cluster(m - b, w, di, G, R, o.panel_rows, &use_reg, o.panel_kernel == 3);
      // panel_kernel 1 is the cluster panel or nothing: the grid panel's
      // mailboxes may not exist in the workspace (the allocation-free path
      // lays them out with zero size)
      if (!use_cluster && o.panel_kernel == 1) return kInvalidArgument;
      if (!use_small && !use_cluster && !plan_panel(m - b, w, o.panel_rows, di, G, R))
        return kInvalidArgument;
      const bool enqueue = la && (use_cluster || use_small);
      if (!enqueue && unread) {
        // a synchronous panel follows enqueued ones: settle them first
        if (int err = read_state(hs, ws, st)) return err;
        if (hs.status != kOk) return hs.status;
        unread = false;
        if (hs.stop_k >= 0) {
          stop = hs.stop_k;
          break;
        }
      }
      e = b + w;
      if (la && !use_cluster && !use_small) {
        // the cooperative grid needs all its CTAs resident: s2 finishes first
        DP_CHECK_CUDA(cudaEventRecord(sc.next, sc.s2));
        DP_CHECK_CUDA(cudaStreamWaitEvent(st, sc.next, 0));
      }

      PanelParams pp;
      pp.a = a;
      pp.lda = lda;
      pp.m = m;
      pp.begin = b;
      pp.end = e;
      pp.rows_per_cta = R;
      pp.positioned = positioned ? 1 : 0;
      pp.parity = parity;
      pp.max_ctas = ws.max_ctas;
      pp.w_max = ws.w_max;
      pp.threshold = o.threshold;
      pp.ipiv = ws.d_ipiv;
      pp.state = ws.state;
      pp.slots = ws.slots;
      pp.xdata = ws.xdata;
      pp.rowk = ws.rowk;
      pp.swap_block = la ? blk + (b - B) : ws.swap_block;
      pp.swap_extra = la ? ext + 2 * (size_t)(b - B) : ws.swap_extra;
      pp.gated = enqueue ? 1 : 0;
      rec.begin(DP_KFAM_PANEL);
      if (use_small) {
        if (int err = launch_panel_small(pp, st)) return err;
      } else if (use_cluster) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = G;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(G);
        cfg.blockDim = dim3(panel_cluster_threads());
        cfg.dynamicSmemBytes =
            use_reg ? panel_reg_smem_bytes(w, R) : panel_cluster_smem_bytes(w, R);
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        dp::note_launch();
        if (use_reg) {
          void* args[] = {&pp};
          DP_CHECK_CUDA(cudaLaunchKernelExC(&cfg, panel_reg_kernel_for(R), args));
        } else {
          DP_CHECK_CUDA(cudaLaunchKernelEx(&cfg, panel_cluster_kernel, pp));
        }
      } else {
        void* args[] = {&pp};
        dp::note_launch();
        DP_CHECK_CUDA(cudaLaunchCooperativeKernel((const void*)panel_factor_kernel, G,
                                                  kPanelThreadsHost, args, panel_smem_bytes(w, R),
                                                  st));
        parity ^= 1;
      }
      rec.end(panel_flops(m, b, w), 16.0 * (double)(m - b) * w, 1);
      positioned = false;
      if (la) widths.push_back(w);

      if (enqueue) {
        // swaps inside the block, then the rest of the block: both skip
        // themselves if this panel or an earlier one stopped (the swaps of
        // the stopping panel itself still apply)
        // (panels up to laswp_solve_max_width() wide: U12 of the block rows
        // solved by the laswp kernel right after their permutation)
        const bool fused = w <= laswp_solve_max_width();
        rec.begin(DP_KFAM_LASWP);
        launch_laswp(a, lda, b, w, pp.swap_block, pp.swap_extra, ws.state, B, b, e, E, st, b,
                     fused ? e : 0, fused ? E : 0);
        rec.end(fused ? (double)w * (w - 1) * (E - e) : 0.0, 16.0 * 2.0 * w * (double)(E - B - w), 1);
        update_columns(a, lda, m, b, w, e, e, E, st, rec, nullptr, nullptr, 2, stop_word, nullptr,
                       fused);
        DP_CHECK_CUDA(cudaGetLastError());
        unread = true;
        b = e;
        continue;
      }
      if (int err = read_state(hs, ws, st)) return err;
      if (hs.status != kOk) return hs.status;
      const double moved = (double)(hs.block_changed + hs.swap_count);
      // (the laswp kernel also solves the block rows of [e, E) unless the
      // panel stopped, which it reads from the state)
      const bool fused = w <= laswp_solve_max_width();
      rec.begin(DP_KFAM_LASWP);
      if (la) {
        launch_laswp(a, lda, b, w, pp.swap_block, pp.swap_extra, ws.state, B, b, e, E, st, -1,
                     fused ? e : 0, fused ? E : 0);
        rec.end(0.0, 16.0 * moved * (double)(E - B - w), 1);
      } else {
        launch_laswp(a, lda, b, w, ws.swap_block, ws.swap_extra, ws.state, 0, b, e, n, st, -1,
                     fused ? e : 0, fused ? E : 0);
        rec.end(0.0, 16.0 * moved * (double)(n - w), 1);
      }
      if (hs.stop_k >= 0) {
        stop = hs.stop_k;
        break;
      }
      // rest of the outer block (U12 solved by the laswp kernel: no stop)
      update_columns(a, lda, m, b, w, e, e, E, st, rec, nullptr, nullptr, 2, nullptr, nullptr,
                     fused);
      DP_CHECK_CUDA(cudaGetLastError());
      b = e;
    }
    if (unread) {
      if (int err = read_state(hs, ws, st)) return err;
      if (hs.status != kOk) return hs.status;
      if (hs.stop_k >= 0) stop = hs.stop_k;
    }
    if (stop >= 0 && la) {
      // the panel that stopped: the last whose first column is <= stop; the
      // ones after it did nothing
      size_t p = 0;
      b = B;
      while (p + 1 < widths.size() && b + widths[p] <= stop) b += widths[p++];
      e = b + widths[p];
      widths.resize(p + 1);
    }
    if (stop < 0 && !la) {
      // right of the outer block: the O(n^3) update
      inv1 = inv2 = BlockInv{};
      if (E < n) block_inverse(B, E - B, 0, inv1, inv2);
      if (int err = update_columns(a, lda, m, B, E - B, E, E, n, st, rec, mixed_ws,
                                   &ws.state->status, terms, nullptr, &inv2))
        return err;
      DP_CHECK_CUDA(cudaGetLastError());
      B = E;
      continue;
    }
    if (stop < 0) {
      const int NE = std::min(pivots, E + NB);   // the next outer block
      const int NNE = std::min(pivots, NE + NB);  // the block after next
      // s1: the next block's columns, then on to its panels
      if (pending) DP_CHECK_CUDA(cudaStreamWaitEvent(st, sc.next, 0));
      // the left swaps of the previous block have read their lists, whose
      // buffer the next block's panels reuse
      DP_CHECK_CUDA(cudaStreamWaitEvent(st, sc.ldone, 0));
      inv1 = inv2 = BlockInv{};
      if (E < n) {
        // T of this block goes to the buffer of two blocks ago, whose last
        // reader is that block's update on the trailing stream: the wait
        // above follows it; without one, wait for the trailing stream here
        if (!pending) {
          DP_CHECK_CUDA(cudaEventRecord(sc.next, sc.s2));
          DP_CHECK_CUDA(cudaStreamWaitEvent(st, sc.next, 0));
        }
        block_inverse(B, E - B, half, inv1, inv2);
      }
      if (int err = apply_deferred(a, lda, blk, ext, B, widths, E, NE, NE, NE, st, rec))
        return err;
      // (mixed precision: its own BF16 scratch, the trailing stream uses ws.mixed)
      if (int err = update_columns(a, lda, m, B, E - B, E, E, NE, st, rec,
                                   terms ? ws.mixed1 : nullptr, &ws.state->status, terms, nullptr,
                                   &inv1))
        return err;
      DP_CHECK_CUDA(cudaGetLastError());
      DP_CHECK_CUDA(cudaEventRecord(sc.block, st));
      // (s2's work so far ends with the previous block's trailing update)
      DP_CHECK_CUDA(cudaEventRecord(sc.tdone, sc.s2));
      // s2: everything else, behind the block
      DP_CHECK_CUDA(cudaStreamWaitEvent(sc.s2, sc.block, 0));
      if (int err = apply_deferred(a, lda, blk, ext, B, widths, NE, n, n, n, sc.s2, *sc.r2))
        return err;
      // s3: the block's swaps on the finished columns left of it, once the
      // previous block's trailing update has read its L columns
      DP_CHECK_CUDA(cudaStreamWaitEvent(sc.s3, sc.block, 0));
      DP_CHECK_CUDA(cudaStreamWaitEvent(sc.s3, sc.tdone, 0));
      if (int err = apply_deferred(a, lda, blk, ext, B, widths, 0, B, B, B, sc.s3, *sc.r3))
        return err;
      DP_CHECK_CUDA(cudaEventRecord(sc.ldone, sc.s3));
      pending = false;
      if (NNE > NE) {
        if (int err = update_columns(a, lda, m, B, E - B, E, NE, NNE, sc.s2, *sc.r2, mixed_ws,
                                     ws.aux_status, terms, nullptr, &inv2))
          return err;
        DP_CHECK_CUDA(cudaEventRecord(sc.next, sc.s2));
        pending = true;
      }
      if (int err = update_columns(a, lda, m, B, E - B, E, std::max(NE, NNE), n, sc.s2, *sc.r2,
                                   mixed_ws, ws.aux_status, terms, nullptr, &inv2))
        return err;
      DP_CHECK_CUDA(cudaGetLastError());
      half ^= 1;
      B = E;
      continue;
    }

    // Stopped at k inside panel [b, e): materialize, then search.
    const int k = stop;
    if (la) {
      // s2 and s3 drain; the block's kept swaps reach every column outside it
      DP_CHECK_CUDA(cudaEventRecord(sc.next, sc.s2));
      DP_CHECK_CUDA(cudaStreamWaitEvent(st, sc.next, 0));
      DP_CHECK_CUDA(cudaEventRecord(sc.ldone, sc.s3));
      DP_CHECK_CUDA(cudaStreamWaitEvent(st, sc.ldone, 0));
      pending = false;
      if (int err = apply_deferred(a, lda, blk, ext, B, widths, 0, B, E, n, st, rec)) return err;
    }
    update_columns(a, lda, m, b, k - b, k, e, E, st, rec);  // rest of the outer block
    // (the trailing stream has drained: its buffers are free)
    inv1 = inv2 = BlockInv{};
    if (E < n) block_inverse(B, k - B, half, inv1, inv2);
    if (int err = update_columns(a, lda, m, B, k - B, k, E, n, st, rec, mixed_ws,
                                 &ws.state->status, terms, nullptr,
                                 &inv2))  // right of the outer block
      return err;
    rec.begin(DP_KFAM_SEARCH);
    if (o.policy == DP_POLICY_NONZERO_COLUMN)
      launch_search_nonzero_column(a, lda, m, n, k, o.threshold, ws.state, st);
    else
      launch_search_active(a, lda, m, n, k, ws.state, ws.cands, kMaxSearchBlocks, st);
    rec.end(0.0, 8.0 * (double)(m - k) * (double)(n - k),
            o.policy == DP_POLICY_NONZERO_COLUMN ? 2 : 1);
    DP_CHECK_CUDA(cudaGetLastError());
    if (int err = read_state(hs, ws, st)) return err;
    if (hs.status != kOk) return hs.status;
    const Cand c = hs.fallback;
    if (!(c.val > o.threshold)) {
      info = k;  // the whole active submatrix is delayed
      break;
    }
    rec.begin(DP_KFAM_SWAP);
    launch_set_record(ws.d_ipiv, ws.d_jpiv, k, c.row, c.col, st);
    launch_swap_row(a, lda, n, k, c.row, st);
    launch_swap_col(a, lda, m, k, c.col, st);
    rec.end(0.0, 32.0 * ((c.row != k ? (double)n : 0.0) + (c.col != k ? (double)m : 0.0)),
            1 + (c.row != k) + (c.col != k));
    DP_CHECK_CUDA(cudaGetLastError());
    if (la) DP_CHECK_CUDA(cudaMemsetAsync(stop_word, 0xFF, sizeof(int), st));  // re-arm
    B = k;
    positioned = true;
  }
  return kOk;
}

bool matrix_byte_count(int lda, int n, size_t& bytes) {
  const size_t cols = (size_t)n, ld = (size_t)lda;
  if (cols != 0 && ld > std::numeric_limits<size_t>::max() / cols) return false;
  const size_t el = ld * cols;
  if (el > std::numeric_limits<size_t>::max() / sizeof(double)) return false;
  bytes = el * sizeof(double);
  return true;
}

// delayed_lu_cuda/delayed_dgetrf_cuda.cu:385-397
bool valid_arguments(int m, int n, const double* a, int lda, const int* ipiv, const int* jpiv) {
  if (m < 0 || n < 0 || lda < std::max(1, m)) return false;
  const int pivots = std::min(m, n);
  if ((m > 0 && n > 0 && a == nullptr) || (pivots > 0 && (ipiv == nullptr || jpiv == nullptr)))
    return false;
  size_t ignored = 0;
  return matrix_byte_count(lda, n, ignored);
}

// Panel-width tuning table (dp_getrf_autotune): per device and order bucket
// floor(log2 n), the (panel width, outer block) pair the tuner found fastest;
// {0, 0} where untuned.  Used by the entry points when the caller leaves
// both widths automatic.
constexpr int kTuneBuckets = 32;
std::mutex g_tune_mutex;
int g_tune[64][kTuneBuckets][2] = {};

int tune_bucket(int n) {
  int b = 0;
  while (b + 1 < kTuneBuckets && (2LL << b) <= n) ++b;
  return b;
}

void apply_tuned_widths(int pivots, Options& o) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  const int* t = g_tune[dev][tune_bucket(pivots)];
  if (t[0] > 0 && t[1] > 0) {
    o.nb = t[0];
    o.nb_outer = t[1];
  }
}

bool resolve_options(const dp_options* in, Options& o) {
  if (!in) return true;
  if (in->nb < 0 || in->panel_rows < 0) return false;
  if (!(in->threshold >= 0.0)) return false;  // rejects NaN and negatives
  if (in->policy != DP_POLICY_FULL_PIVOT && in->policy != DP_POLICY_NONZERO_COLUMN) return false;
  if (in->nb_outer < 0) return false;
  o.nb = in->nb ? std::min(in->nb, kMaxPanelWidth) : kDefaultNb;
  o.nb_outer = in->nb_outer ? in->nb_outer : std::max(kDefaultNbOuter, o.nb);
  o.threshold = in->threshold;
  o.policy = in->policy;
  o.panel_rows = in->panel_rows ? in->panel_rows : kDefaultPanelRows;
  if (in->panel_kernel < 0 || in->panel_kernel > 3) return false;
  o.panel_kernel = in->panel_kernel;
  if (!valid_precision(in->precision))
    return false;
  o.precision = in->precision;
  if (in->lookahead < 0 || in->lookahead > 2) return false;
  o.lookahead = in->lookahead;
  return true;
}

}  // namespace

int getrf_device(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                 cudaStream_t st, const dp_options* opt) {
  clear_report();
  if (info == nullptr) return kInvalidArgument;
  *info = -1;
  Options o;
  if (!valid_arguments(m, n, d_a, lda, ipiv, jpiv) || !resolve_options(opt, o))
    return kInvalidArgument;
  const int pivots = std::min(m, n);
  if (!opt || (opt->nb == 0 && opt->nb_outer == 0)) apply_tuned_widths(pivots, o);
  *info = pivots;
  for (int k = 0; k < pivots; ++k) ipiv[k] = jpiv[k] = k;
  if (pivots == 0) {
    g_report.info = 0;
    return kOk;
  }

  DeviceInfo di;
  if (device_info(di) != kOk) {
    *info = -1;
    return kCudaFailure;
  }
  Workspace ws;
  const int w_max = kMaxPanelWidth;
  const size_t mixed_bytes = mixed_terms(o.precision)
                                 ? mixed_scratch_bytes(m, n, std::max(o.nb_outer, o.nb),
                                                       mixed_terms(o.precision))
                                 : 0;
  const int NB = std::max(o.nb_outer, o.nb);
  Lanes* lanes = nullptr;
  if (o.lookahead == 1 || (o.lookahead == 0 && pivots > NB)) lanes = lanes_for_device();
  const int defer_cap = lanes ? std::min(NB, pivots) : 0;
  const size_t mixed1_bytes =
      lanes && mixed_terms(o.precision) ? mixed_scratch_bytes(m, NB, NB, mixed_terms(o.precision))
                                        : 0;
  InvPlan ip;  // outer blocks wider than the TRSM kernel's are solved by inverse
  if (g_block_solve.load() != 2 && NB > trsm_max_width() && NB <= lower_inverse_max_width() &&
      n > NB) {
    ip.ld = NB;
    ip.copy1_cols = lanes ? NB : 0;
    ip.copy2_cols = n;
  }
  const size_t bytes = layout_workspace(ws, nullptr, pivots, di.sms, w_max, mixed_bytes,
                                        defer_cap, mixed1_bytes, ip);
  char* base = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&base), bytes, st) != cudaSuccess) {
    cudaGetLastError();
    *info = -1;
    return kAllocationFailed;
  }
  layout_workspace(ws, base, pivots, di.sms, w_max, mixed_bytes, defer_cap, mixed1_bytes, ip);
  int status = kOk;
  // the scratch regions (at the end) are fully written before use; clear the rest
  const size_t clear = (size_t)(ws.scratch - base);
  if (cudaMemsetAsync(base, 0, clear, st) != cudaSuccess) status = kCudaFailure;
  int inf = pivots;
  HostTrace trace;
  g_trace = &trace;
  Schedule sc;
  sc.s1 = lanes ? lanes->panel : st;
  sc.s2 = lanes ? lanes->trail : nullptr;
  sc.s3 = lanes ? lanes->left : nullptr;
  Recorder rec(sc.s1), rec2(lanes ? lanes->trail : st), rec3(lanes ? lanes->left : st);
  sc.r1 = &rec;
  sc.r2 = &rec2;
  sc.r3 = &rec3;
  rec2.lane = 1;
  rec3.lane = 2;
  cudaEvent_t tl_base = nullptr;
  if (rec.on && timeline_path()) {
    tl_base = event_get();
    cudaEventRecord(tl_base, st);
    rec.base = rec2.base = rec3.base = tl_base;
  }
  if (lanes) {
    sc.block = lanes->block;
    sc.next = lanes->next;
    sc.ldone = lanes->ldone;
    sc.tdone = lanes->tdone;
    if (status == kOk && (cudaEventRecord(lanes->fork, st) != cudaSuccess ||
                          cudaStreamWaitEvent(lanes->panel, lanes->fork, 0) != cudaSuccess ||
                          cudaStreamWaitEvent(lanes->trail, lanes->fork, 0) != cudaSuccess ||
                          cudaStreamWaitEvent(lanes->left, lanes->fork, 0) != cudaSuccess ||
                          cudaEventRecord(lanes->ldone, lanes->left) != cudaSuccess))
      status = kCudaFailure;
  }
  if (status == kOk) status = factorize(m, n, d_a, lda, o, ws, di, sc, inf);
  int aux = kOk;
  if (lanes) {
    // st waits for every lane whatever happened, before the workspace is freed
    cudaEventRecord(lanes->join, lanes->panel);
    cudaStreamWaitEvent(st, lanes->join, 0);
    cudaEventRecord(lanes->join, lanes->trail);
    cudaStreamWaitEvent(st, lanes->join, 0);
    cudaEventRecord(lanes->join, lanes->left);
    cudaStreamWaitEvent(st, lanes->join, 0);
    if (status == kOk &&
        cudaMemcpyAsync(&aux, ws.aux_status, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess)
      status = kCudaFailure;
  }
  State fin{};
  if (status == kOk) {
    if (cudaMemcpyAsync(ipiv, ws.d_ipiv, sizeof(int) * pivots, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(jpiv, ws.d_jpiv, sizeof(int) * pivots, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(&fin, ws.state, sizeof(State), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      status = kCudaFailure;
  }
  cudaFreeAsync(base, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && status == kOk) status = kCudaFailure;
  if (status == kOk && aux != kOk) status = aux;
  rec.flush(status == kOk);
  rec2.flush(status == kOk);
  rec3.flush(status == kOk);
  if (tl_base) {
    std::lock_guard<std::mutex> lock(g_stats_mutex);
    ++g_timeline_calls;
    event_put(tl_base);
  }
  g_trace = nullptr;
  if (status != kOk) {
    cudaGetLastError();
    *info = -1;
    return status;
  }
  *info = inf;
  set_report(fin, inf);
  return kOk;
}

int getrf_host(int m, int n, double* a, int lda, int* ipiv, int* jpiv, int* info,
               cudaStream_t st, const dp_options* opt) {
  clear_report();
  if (info == nullptr) return kInvalidArgument;
  *info = -1;
  if (!valid_arguments(m, n, a, lda, ipiv, jpiv)) return kInvalidArgument;
  const int pivots = std::min(m, n);
  if (pivots == 0) {  // delayed_dgetrf_cuda.cu:456-460
    *info = 0;
    g_report.info = 0;
    return kOk;
  }
  size_t bytes = 0;
  if (!matrix_byte_count(lda, n, bytes)) return kInvalidArgument;
  double* d_a = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&d_a), bytes, st) != cudaSuccess) {
    cudaGetLastError();
    return kAllocationFailed;
  }
  int status = kOk;
  if (cudaMemcpyAsync(d_a, a, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) status = kCudaFailure;
  if (status == kOk) status = getrf_device(m, n, d_a, lda, ipiv, jpiv, info, st, opt);
  if (status == kOk) {
    if (cudaMemcpyAsync(a, d_a, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      *info = -1;
      status = kCudaFailure;
      clear_report();
    }
  }
  cudaFreeAsync(d_a, st);
  cudaStreamSynchronize(st);
  if (status != kOk) cudaGetLastError();
  return status;
}

// ------------------------------------------- allocation-free variant ----
// Some callers must not allocate device memory during a call: code running
// under a memory manager that owns the whole device pool, callers that
// budget every byte of HBM up front, or processes whose allocator is not the
// CUDA runtime's.  getrf_device_noalloc runs the same plain-FP64 delayed LU
// as getrf_device but takes its scratch (state block, device swap records,
// panel swap lists, fallback-search candidates) from one file-scope device
// array instead of cudaMallocAsync.  It always uses the cluster panel, which
// needs no cross-CTA mailboxes, so the scratch stays small.
//
// The array belongs to the library: every GPU that loads it holds
// kNoallocScratchBytes for as long as the process lives, every call uses the
// same array (calls that overlap on the GPU - other threads or other streams
// - race with each other and must be serialised by the caller), and each call
// clears what it needs at start.  Limits: at most kNoallocMaxPivots pivots,
// and the tallest panel must fit the cluster panel kernel.
constexpr int kNoallocMaxPivots = 32768;
constexpr size_t kNoallocScratchBytes = 320 * 1024;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Device address of g_noalloc_scratch per device, looked up once (the host
// name of a __device__ array is only a host-side handle, never a device
// address).  The lookup is a host-side query and allocates nothing; it runs
// on the first call on each device.  The entry point reads the pivot state
// from the device during the call and synchronises its stream before it
// returns, as every getrf entry point does.
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[64] = {};

int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return kCudaFailure;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return kCudaFailure;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return kOk;
}

int getrf_device_noalloc(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                         cudaStream_t st) {
  clear_report();
  if (info == nullptr) return kInvalidArgument;
  *info = -1;
  if (!valid_arguments(m, n, d_a, lda, ipiv, jpiv)) return kInvalidArgument;
  const int pivots = std::min(m, n);
  if (pivots > kNoallocMaxPivots) return kInvalidArgument;  // beyond the fixed scratch
  Options o;
  o.panel_kernel = 1;  // cluster panel only: no mailbox scratch
  DeviceInfo di;
  if (pivots > 0 && device_info(di) != kOk) return kCudaFailure;
  if (pivots > 0) {
    // the first panel is the tallest; every later one fits if it does
    int w = std::min(o.nb, pivots), C = 0, R = 0;
    if (!plan_cluster(m, w, di, C, R)) return kInvalidArgument;
  }
  *info = pivots;
  for (int k = 0; k < pivots; ++k) ipiv[k] = jpiv[k] = k;
  if (pivots == 0) {
    g_report.info = 0;
    return kOk;
  }

  void* scratch = nullptr;
  if (noalloc_scratch(&scratch) != kOk) {
    *info = -1;
    return kCudaFailure;
  }
  Workspace ws;
  const size_t bytes = layout_workspace(ws, nullptr, pivots, 0, kMaxPanelWidth, 0);
  if (bytes > kNoallocScratchBytes) {
    *info = -1;
    return kInvalidArgument;
  }
  char* base = static_cast<char*>(scratch);
  layout_workspace(ws, base, pivots, 0, kMaxPanelWidth, 0);
  int status = kOk;
  if (cudaMemsetAsync(base, 0, bytes, st) != cudaSuccess) status = kCudaFailure;
  int inf = pivots;
  Recorder rec(st);
  rec.on = false;  // no timing events on this path
  Schedule sc;  // one stream: no look-ahead
  sc.s1 = st;
  sc.r1 = &rec;
  sc.r2 = &rec;
  sc.r3 = &rec;
  if (status == kOk) status = factorize(m, n, d_a, lda, o, ws, di, sc, inf);
  State fin{};
  if (status == kOk) {
    if (cudaMemcpyAsync(ipiv, ws.d_ipiv, sizeof(int) * pivots, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(jpiv, ws.d_jpiv, sizeof(int) * pivots, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(&fin, ws.state, sizeof(State), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      status = kCudaFailure;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess && status == kOk) status = kCudaFailure;
  if (status != kOk) {
    cudaGetLastError();
    *info = -1;
    return status;
  }
  *info = inf;
  set_report(fin, inf);
  return kOk;
}

}  // namespace dp

// ---------------------------------------------------------------- C ABI ----
extern "C" {

void dp_options_init(dp_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->nb = 64;
  opt->threshold = 0.0;
  opt->policy = DP_POLICY_FULL_PIVOT;
  opt->panel_rows = 0;
}

int dp_getrf_device_ex(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                       void* stream, const dp_options* opt) {
  return dp::getrf_device(m, n, d_a, lda, ipiv, jpiv, info, static_cast<cudaStream_t>(stream), opt);
}

int dp_getrf_device(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                    void* stream) {
  return dp::getrf_device(m, n, d_a, lda, ipiv, jpiv, info, static_cast<cudaStream_t>(stream),
                          nullptr);
}

int dp_getrf_host(int m, int n, double* a, int lda, int* ipiv, int* jpiv, int* info,
                  void* stream) {
  return dp::getrf_host(m, n, a, lda, ipiv, jpiv, info, static_cast<cudaStream_t>(stream), nullptr);
}

int dp_getrf_native_device(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                           void* stream) {
  return dp_getrf_device(m, n, d_a, lda, ipiv, jpiv, info, stream);
}
int dp_getrf_native_host(int m, int n, double* a, int lda, int* ipiv, int* jpiv, int* info,
                         void* stream) {
  return dp_getrf_host(m, n, a, lda, ipiv, jpiv, info, stream);
}
int dp_getrf_hybrid_device(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                           void* stream) {
  return dp_getrf_device(m, n, d_a, lda, ipiv, jpiv, info, stream);
}
int dp_getrf_hybrid_host(int m, int n, double* a, int lda, int* ipiv, int* jpiv, int* info,
                         void* stream) {
  return dp_getrf_host(m, n, a, lda, ipiv, jpiv, info, stream);
}

int dp_block_solve(int mode) {
  if (mode < 0 || mode > 2) return -1;
  return dp::g_block_solve.exchange(mode);
}

int dp_getrf_last_report(dp_getrf_report* out) {
  if (!out) return DP_INVALID_ARGUMENT;
  *out = dp::g_report;
  return DP_SUCCESS;
}

int dp_getrf_autotune(int n, int* nb, int* nb_outer, void* stream) {
  if (n < 1 || n > 65536) return DP_INVALID_ARGUMENT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DP_CUDA_FAILURE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  static const int kCand[][2] = {{32, 64},  {64, 64},   {32, 128}, {64, 128},
                                 {128, 128}, {32, 256}, {64, 256}, {128, 256}};
  const size_t elems = (size_t)n * n;
  double *src = nullptr, *work = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&src), sizeof(double) * elems, st) != cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&work), sizeof(double) * elems, st) !=
          cudaSuccess) {
    cudaGetLastError();
    if (src) cudaFreeAsync(src, st);
    cudaStreamSynchronize(st);
    return DP_ALLOCATION_FAILED;
  }
  dp::launch_fill_normal(src, (long long)elems, 0x5eed0000ull + (unsigned long long)n, st);
  std::vector<int> ipiv(n), jpiv(n);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess
               ? DP_SUCCESS
               : DP_CUDA_FAILURE;
  float best = 1e30f;
  int bnb = 0, bNB = 0;
  for (const auto& c : kCand) {
    if (rc != DP_SUCCESS) break;
    if (c[1] > n && c[1] != 64) continue;  // an outer block beyond the order changes nothing
    dp_options o;
    dp_options_init(&o);
    o.nb = c[0];
    o.nb_outer = c[1];
    float t = 1e30f;
    for (int rep = 0; rep < 2 && rc == DP_SUCCESS; ++rep) {
      int info = -1;
      if (cudaMemcpyAsync(work, src, sizeof(double) * elems, cudaMemcpyDeviceToDevice, st) !=
              cudaSuccess ||
          cudaEventRecord(e0, st) != cudaSuccess) {
        rc = DP_CUDA_FAILURE;
        break;
      }
      rc = dp::getrf_device(n, n, work, n, ipiv.data(), jpiv.data(), &info, st, &o);
      float ms = 0.f;
      if (rc == DP_SUCCESS && (cudaEventRecord(e1, st) != cudaSuccess ||
                               cudaEventSynchronize(e1) != cudaSuccess ||
                               cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        rc = DP_CUDA_FAILURE;
      t = std::min(t, ms);
    }
    if (rc == DP_SUCCESS && t < best) {
      best = t;
      bnb = c[0];
      bNB = c[1];
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFreeAsync(src, st);
  cudaFreeAsync(work, st);
  cudaStreamSynchronize(st);
  if (rc != DP_SUCCESS) return rc;
  {
    std::lock_guard<std::mutex> lock(dp::g_tune_mutex);
    dp::g_tune[dev][dp::tune_bucket(n)][0] = bnb;
    dp::g_tune[dev][dp::tune_bucket(n)][1] = bNB;
  }
  if (nb) *nb = bnb;
  if (nb_outer) *nb_outer = bNB;
  return DP_SUCCESS;
}

int dp_getrf_tune_save(const char* path) {
  int dev = 0;
  if (!path || cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return DP_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "w");
  if (!f) return DP_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(dp::g_tune_mutex);
    for (int b = 0; b < dp::kTuneBuckets; ++b)
      if (dp::g_tune[dev][b][0] > 0)
        std::fprintf(f, "%lld %lld %d %d\n", 1LL << b, (2LL << b) - 1, dp::g_tune[dev][b][0],
                     dp::g_tune[dev][b][1]);
  }
  return std::fclose(f) == 0 ? DP_SUCCESS : DP_INVALID_ARGUMENT;
}

int dp_getrf_tune_load(const char* path) {
  int dev = 0;
  if (!path || cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return DP_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "r");
  if (!f) return DP_INVALID_ARGUMENT;
  int table[dp::kTuneBuckets][2] = {};
  long long lo = 0, hi = 0;
  int nb = 0, NB = 0, rc = DP_SUCCESS;
  while (true) {
    const int got = std::fscanf(f, "%lld %lld %d %d", &lo, &hi, &nb, &NB);
    if (got == EOF) break;
    const int b = lo >= 1 ? dp::tune_bucket((int)std::min<long long>(lo, 1 << 30)) : -1;
    if (got != 4 || b < 0 || (1LL << b) != lo || hi != (2LL << b) - 1 || nb < 1 ||
        nb > dp::kMaxPanelWidth || NB < nb) {
      rc = DP_INVALID_ARGUMENT;
      break;
    }
    table[b][0] = nb;
    table[b][1] = NB;
  }
  std::fclose(f);
  if (rc != DP_SUCCESS) return rc;
  std::lock_guard<std::mutex> lock(dp::g_tune_mutex);
  std::memcpy(dp::g_tune[dev], table, sizeof(table));
  return DP_SUCCESS;
}

void dp_stats_enable(int on) {
  std::lock_guard<std::mutex> lock(dp::g_stats_mutex);
  dp::g_stats_on = on != 0;
}

unsigned dp_stats_families(unsigned mask) {
  std::lock_guard<std::mutex> lock(dp::g_stats_mutex);
  const unsigned prev = dp::g_stats_mask;
  dp::g_stats_mask = mask;
  return prev;
}

void dp_stats_reset(void) {
  std::lock_guard<std::mutex> lock(dp::g_stats_mutex);
  std::memset(&dp::g_stats, 0, sizeof(dp::g_stats));
}

void dp_stats_get(dp_kernel_stats* out) {
  if (!out) return;
  std::lock_guard<std::mutex> lock(dp::g_stats_mutex);
  *out = dp::g_stats;
}

int dp_getrf_device_noalloc(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                            void* stream) {
  return dp::getrf_device_noalloc(m, n, d_a, lda, ipiv, jpiv, info,
                                  static_cast<cudaStream_t>(stream));
}

const char* dp_status_string(int status) {
  switch (status) {
    case DP_SUCCESS: return "success";
    case DP_INVALID_ARGUMENT: return "invalid argument";
    case DP_ALLOCATION_FAILED: return "CUDA allocation failed";
    case DP_CUDA_FAILURE: return "CUDA runtime failure";
    case DP_LIBRARY_FAILURE: return "cuBLAS failure";
    case DP_DEVICE_TIMEOUT: return "device wait timed out";
  }
  return "unknown status";
}

}  // extern "C"

// ------------------------------------------------ C++ drop-in symbols ----
namespace {
DelayedGetrfCudaStatus to_status(int s) { return static_cast<DelayedGetrfCudaStatus>(s); }
}  // namespace

DelayedGetrfCudaStatus delayed_getrf_cuda_device(int m, int n, double* d_a, int lda, int* ipiv,
                                                 int* jpiv, int& info, cudaStream_t stream) {
  return to_status(dp::getrf_device(m, n, d_a, lda, ipiv, jpiv, &info, stream, nullptr));
}
DelayedGetrfCudaStatus delayed_getrf_cuda_host(int m, int n, double* a, int lda, int* ipiv,
                                               int* jpiv, int& info, cudaStream_t stream) {
  return to_status(dp::getrf_host(m, n, a, lda, ipiv, jpiv, &info, stream, nullptr));
}
DelayedGetrfCudaStatus delayed_getrf_cuda_native_device(int m, int n, double* d_a, int lda,
                                                        int* ipiv, int* jpiv, int& info,
                                                        cudaStream_t stream) {
  return delayed_getrf_cuda_device(m, n, d_a, lda, ipiv, jpiv, info, stream);
}
DelayedGetrfCudaStatus delayed_getrf_cuda_native_host(int m, int n, double* a, int lda, int* ipiv,
                                                      int* jpiv, int& info, cudaStream_t stream) {
  return delayed_getrf_cuda_host(m, n, a, lda, ipiv, jpiv, info, stream);
}
DelayedGetrfCudaStatus delayed_getrf_cuda_hybrid_device(int m, int n, double* d_a, int lda,
                                                        int* ipiv, int* jpiv, int& info,
                                                        cudaStream_t stream) {
  return delayed_getrf_cuda_device(m, n, d_a, lda, ipiv, jpiv, info, stream);
}
DelayedGetrfCudaStatus delayed_getrf_cuda_hybrid_host(int m, int n, double* a, int lda, int* ipiv,
                                                      int* jpiv, int& info, cudaStream_t stream) {
  return delayed_getrf_cuda_host(m, n, a, lda, ipiv, jpiv, info, stream);
}
const char* delayed_getrf_cuda_status_string(DelayedGetrfCudaStatus status) {
  return dp_status_string(static_cast<int>(status));
}

extern "C" long long dp_kernel_launches(void) { return dp::g_kernel_launches.load(); }
