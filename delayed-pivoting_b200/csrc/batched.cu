// Batched delayed-pivoting LU: thousands of independent square matrices of
// uneven sizes (n <= 512) in one persistent launch.
//
// Semantics per matrix are those of delayed_lu/delayed_dgetrf.cpp:129-251
// (column partial pivoting, acceptance |alpha| > threshold, full-pivot
// fallback on a column without an acceptable pivot after bringing the far
// columns up to date, delay when the whole active block has none, swap
// histories, compact L\U in place).  Blocking only changes rounding, so the
// records equal the single-matrix path's and the reference's.
//
// One CTA of 256 threads factors one matrix at a time; CTAs pull matrix
// indices from a device work queue ordered largest first, so the tail is
// short.  Per panel of nb <= 32 columns:
//   panel      the n - b panel rows live in REGISTERS, two rows per thread,
//              thread t owning panel rows t and t + 256 for the whole panel,
//              factored in sub-panels of 8 columns with a rank-8 update of
//              the rest of the register window after each.  A row swap only
//              exchanges the logical positions the owners keep (no data
//              moves); the candidate for column s + 1 is taken while column
//              s + 1 is updated, each warp's winning lane pushes its row into
//              shared memory, and ONE barrier per column publishes the warp
//              winners - every thread then knows the pivot row and reads it
//              from shared memory.  Ties go to the smaller logical row, NaN
//              never wins (delayed_dgetrf_cuda.cu:13-20, :46).
//   write-back the panel, in logical row order, to the matrix and to shared
//              memory (L11 and L21 for the update)
//   permute    the panel's composite row permutation (at most 2 nb rows move)
//              on every column outside it, four lanes per column gathering
//              the moved rows into registers before storing them
//   update     per 256 trailing columns: U12 = L11^{-1} A12 (one thread per
//              column, in registers) written to the matrix and to a shared
//              tile, then A22 -= L21 U12 on the FP64 tensor path (mma.sync
//              m16n8k4, warp tiles 32 x 32, C prefetched into registers
//              before the k-loop)
//   fallback   materialize the far columns with the executed prefix, 2-D
//              argmax (smaller column, then smaller row on ties), full-row and
//              full-column swaps, restart the panel at k with the pivot placed
// The panel width is chosen per size bucket (dp_batch_options.nb_bucket);
// dp_batch_autotune fills that table by timing the candidates.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_bf16.h>

#include "delayed_pivoting_b200.h"
#include "dp_device.cuh"
#include "dp_kernels.h"
#include "serve_kernels.h"

namespace dp {
namespace batch {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRpt = 2;                   // panel rows per thread
constexpr int kMaxN = kThreads * kRpt;    // 512
constexpr int kMaxNb = 32;                // panel width limit = register window
constexpr int kSb = 8;                    // sub-panel width inside the window
constexpr int kTileM = 64;                // trailing update tile: 8 warps as 2 x 4,
constexpr int kTileN = 128;               // warp tile 32 x 32
constexpr int kStageN = 2 * kTileN;       // trailing columns solved per staging round
constexpr int kLdb = 36;                  // shared U12 tile stride (== 4 mod 16)
constexpr int kLdsave = kMaxNb + 2;
constexpr int kNone = INT_MAX;            // logical position of a thread's missing row
static_assert(kMaxN == DP_BATCH_MAX_N, "batched kernel covers n <= DP_BATCH_MAX_N");
static_assert(kMaxNb == DP_BATCH_MAX_NB, "panel width limit");
static_assert(kStageN == kThreads, "one staging column per thread");

struct Params {
  double* base;
  const long long* offsets;      // first element of matrix i (lda = n_i)
  const int* ns;                 // order of matrix i
  const long long* rec_offsets;  // first record of matrix i
  const int* order;              // processing order (largest first)
  int count;
  int* queue;                    // work counter, zeroed before the launch
  int* ipiv;
  int* jpiv;
  int* info;
  unsigned long long* ties;      // near-tie detector: decisions checked, order-sensitive
                                 // ones, bits of the largest runner-up / winner ratio
  double threshold;
  int nb_bucket[DP_BATCH_BUCKETS];
  int pr;                        // column stride of the shared panel
};

__host__ __device__ constexpr int panel_ld(int rows) {
  // >= rows and == 4 (mod 16) doubles: the DMMA A fragments read from the
  // panel are conflict-free
  return ((rows + 11) / 16) * 16 + 4;
}

__host__ __device__ inline int bucket_of(int n) {
  return n < 64 ? 0 : n < 128 ? 1 : n < 256 ? 2 : 3;
}

struct Smem {
  // dynamic part: P [pr * kMaxNb], then Bs [kStageN * kLdb]
  double crow[2][kWarps][kSb + 1]; // each warp's candidate row (sub-panel part) and the
                                   // reciprocal of its pivot entry, by step parity
  double rval[2][kWarps];          // each warp's best magnitude (>= 0) and logical row
  int rkey[2][kWarps];
  double rsec[2][kWarps];          // each warp's runner-up magnitude (near-tie detector)
  double psave[kSb][kLdsave];      // the current sub-panel's pivot rows, whole window
  short mv_dst[2 * kMaxNb];        // the panel's composite row permutation:
  short mv_src[2 * kMaxNb];        // panel row mv_src[j] moves to mv_dst[j]
  int mv_count;
  double fval[kWarps];             // fallback search
  double fsec[kWarps];
  int frow[kWarps];
  int fcol[kWarps];
  int slot;
};

__device__ __forceinline__ void mma_f64(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// Mixed form of the trailing update: BF16 pieces x = x1 + x2 [+ x3] (each the
// BF16 rounding of what the earlier ones left, as in the single-matrix
// tensor-core update), products of pieces (i, j) with i + j <= TERMS - 1 on
// mma.sync.m16n8k16 with FP32 accumulation.
template <int TERMS>
__device__ __forceinline__ void split_pieces(double x, __nv_bfloat16 (&piece)[TERMS]) {
#pragma unroll
  for (int t = 0; t < TERMS; ++t) {
    piece[t] = __double2bfloat16(x);
    x -= (double)__bfloat162float(piece[t]);
  }
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4],
                                         const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Candidate (magnitude v, logical row key) beats (cv, ck)?
__device__ __forceinline__ bool beats(double v, int key, double cv, int ck) {
  return v > cv || (v == cv && key < ck);
}

// Best (largest magnitude, then smallest key) of the warp's candidates.  A
// magnitude is >= 0 (a lane without a candidate offers 0 with key kNone), so
// its bit pattern orders like its value: max of the high word, then of the
// low word among the lanes holding that high word, then min key among the
// lanes holding the maximum - three warp reductions.
__device__ __forceinline__ void warp_best(double v, int key, double& bv, int& bk) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(u >> 32), lo = (unsigned)u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  bk = __reduce_min_sync(0xffffffffu, (hi == mhi && lo == mlo) ? key : kNone);
  bv = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

// Largest of the lanes' non-negative magnitudes (bit-pattern order).
__device__ __forceinline__ double warp_max_pos(double v) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(u >> 32), lo = (unsigned)u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  return __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

// Offers candidate (v, key) to a running best (cv, ck) with runner-up cs:
// the magnitude that does not win becomes a runner-up candidate.
__device__ __forceinline__ bool offer(double v, int key, double& cv, int& ck, double& cs) {
  if (beats(v, key, cv, ck)) {
    cs = fmax(cs, cv);
    cv = v;
    ck = key;
    return true;
  }
  cs = fmax(cs, v);
  return false;
}

// Counts one pivot decision of step k in the batch's near-tie counters.
__device__ __forceinline__ void note_tie(unsigned long long* ties, int k, double best,
                                         double second) {
  atomicAdd(ties, 1ull);
  if (best > 0.0) {
    if (best - second <= kNearTieC * (double)(k + 1) * 0x1p-53 * best) atomicAdd(ties + 1, 1ull);
    atomicMax(ties + 2, (unsigned long long)__double_as_longlong(second / best));
  }
}

// Factor panel columns [b, b + w) of the n x n matrix A (rows b..n-1).
// Returns the first step without an acceptable pivot (-1: all w steps done).
// Writes the panel back in logical row order to A and to P (column stride
// pr), the step pivots to ipiv, and the rows that moved to s.mv_*.
//
// Thread t owns panel rows t and t + 256 (physical rows) and keeps a window
// of 32 of their columns in registers, x[i][c] = panel column base + c.  The
// window is factored in sub-panels of kSb columns: kSb unrolled steps of
// rank-1 updates confined to the sub-panel (one barrier each), then the
// sub-panel's pivot rows are solved for the rest of the window (U12 =
// L11^{-1} A12, in shared memory) and the remaining rows take one rank-kSb
// update; finished columns go to P in physical row order and the window
// shifts by kSb.  The compiled step body is one sub-panel long.
__device__ __forceinline__ int panel_regs(double* A, int n, int lda, int b, int w,
                                          bool positioned, double thr, double* P, int pr,
                                          Smem& s, int* ipiv, unsigned long long* ties) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int rows = n - b;
  double x[kRpt][kMaxNb];
  int lp[kRpt];
#pragma unroll
  for (int i = 0; i < kRpt; ++i) {
    const int r = tid + i * kThreads;
    lp[i] = r < rows ? r : kNone;
#pragma unroll
    for (int c = 0; c < kMaxNb; ++c)
      x[i][c] = (r < rows && c < w) ? A[idx(b + r, b + c, lda)] : 0.0;
  }

  // warp best of the lane candidates (cv >= 0, ck from the lane's row ci);
  // the winning lane pushes its sub-panel columns j.., the reciprocal of its
  // entry in column j (computed by every lane ahead of the reductions, off
  // the path after the barrier) and the warp's result
  auto push = [&](int j, int par, double cv, int ck, int ci, double cs) {
    double pv = 0.0;
#pragma unroll
    for (int c = 0; c < kSb; ++c)
      if (c == j) pv = ci ? x[kRpt - 1][c] : x[0][c];
    const double rinv = 1.0 / pv;
    double wv;
    int wk;
    warp_best(cv, ck, wv, wk);
    // the warp's runner-up: the winner lane's runner-up, every other lane's best
    const double ws = warp_max_pos((wk != kNone && ck == wk) ? cs : (ck != kNone ? cv : cs));
    if (wk != kNone ? ck == wk : lane == 0) {
      if (wk != kNone) {
#pragma unroll
        for (int c = 0; c < kSb; ++c)
          if (c >= j) s.crow[par][warp][c] = ci ? x[kRpt - 1][c] : x[0][c];
        s.crow[par][warp][kSb] = rinv;
      }
      s.rval[par][warp] = wv;
      s.rkey[par][warp] = wk;
      s.rsec[par][warp] = ws;
    }
  };
  // candidate of window column 0 among the rows at logical positions >= first
  auto first_candidate = [&](int first, bool placed) {
    double cv = 0.0, cs = 0.0;
    int ck = kNone, ci = 0;
#pragma unroll
    for (int i = 0; i < kRpt; ++i) {
      if (lp[i] == kNone || lp[i] < first) continue;
      // a placed pivot (after a fallback) is the only candidate of its step
      if (placed && lp[i] != first) continue;
      const double v = placed ? INFINITY : fabs(x[i][0]);
      if (offer(v, lp[i], cv, ck, cs)) ci = i;
    }
    push(0, first & 1, cv, ck, ci, cs);
  };

  first_candidate(0, positioned);
  if (tid == 0) s.mv_count = 0;
  __syncthreads();

  int stop = -1;
  int base = 0;  // panel column of window column 0
  while (base < w) {
    const int sw = min(kSb, w - base);
    int kd = sw;  // steps executed in this sub-panel
#pragma unroll
    for (int j = 0; j < kSb; ++j) {
      if (j >= sw) break;
      const int st = base + j, par = st & 1;
      double bv;
      int bk;
      warp_best(s.rval[par][lane & (kWarps - 1)], s.rkey[par][lane & (kWarps - 1)], bv, bk);
      // the warp that offered the winner (keys of real candidates are unique)
      const int bw = max(0, __ffs(__ballot_sync(0xffffffffu, lane < kWarps && bk != kNone &&
                                                                s.rkey[par][lane] == bk)) - 1);
      const bool placed = positioned && st == 0;
      if (!placed) {
        // runner-up over the warps (lanes >= kWarps repeat lanes < kWarps)
        const int q = lane & (kWarps - 1);
        const double bs = warp_max_pos((bk != kNone && s.rkey[par][q] == bk)
                                           ? s.rsec[par][q]
                                           : (s.rkey[par][q] != kNone ? s.rval[par][q]
                                                                      : s.rsec[par][q]));
        if (tid == 0) note_tie(ties, b + st, bk != kNone ? bv : 0.0, bs);
      }
      if (!placed && !(bv > thr)) {
        stop = st;
        kd = j;
        break;
      }
      const double* prow = s.crow[par][bw];
      const int p = bk;  // logical position of the pivot row before the swap
      if (tid == 0 && !placed) ipiv[b + st] = b + p;
      const double inv = prow[kSb];
      double cv = 0.0, cs = 0.0;
      int ck = kNone, ci = 0;
#pragma unroll
      for (int i = 0; i < kRpt; ++i) {
        if (lp[i] == p) {
          lp[i] = st;  // the pivot row: keep its window for the U12 solve
#pragma unroll
          for (int g = 0; g < kMaxNb / kSb; ++g)
            if (base + g * kSb < w) {
#pragma unroll
              for (int c = g * kSb; c < (g + 1) * kSb; ++c) s.psave[j][c] = x[i][c];
            }
        } else if (lp[i] == st) {
          lp[i] = p;
        }
        if (lp[i] == kNone || lp[i] <= st) continue;
        const double l = x[i][j] * inv;
        x[i][j] = l;
#pragma unroll
        for (int c = j + 1; c < kSb; ++c) x[i][c] = fma(-l, prow[c], x[i][c]);
        if (j + 1 < kSb) {
          const double v = fabs(x[i][j + 1 < kSb ? j + 1 : 0]);
          if (offer(v, lp[i], cv, ck, cs)) ci = i;
        }
      }
      if (j + 1 < sw) {
        push(j + 1, par ^ 1, cv, ck, ci, cs);
        __syncthreads();
      }
    }
    // the window columns right of the sub-panel take its kd executed steps
    const int rest = w - base - kSb;
    __syncthreads();  // psave complete
    if (kd > 0 && rest > 0) {
      for (int c = kSb + tid; c < kSb + rest; c += kThreads)
        for (int j = 1; j < kd; ++j) {
          double u = s.psave[j][c];
          for (int t = 0; t < j; ++t) u = fma(-s.psave[j][t], s.psave[t][c], u);
          s.psave[j][c] = u;
        }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < kRpt; ++i) {
        if (lp[i] == kNone || lp[i] < base) continue;
        if (lp[i] < base + kd) {  // a pivot row of this sub-panel takes its U12 row
          const double* u = s.psave[lp[i] - base];
#pragma unroll
          for (int g = 1; g < kMaxNb / kSb; ++g)
            if (base + g * kSb < w) {
#pragma unroll
              for (int c = g * kSb; c < (g + 1) * kSb; ++c) x[i][c] = u[c];
            }
        } else {
#pragma unroll
          for (int g = 1; g < kMaxNb / kSb; ++g)
            if (base + g * kSb < w) {
#pragma unroll
              for (int t = 0; t < kSb; ++t)
                if (t < kd) {
                  const double l = x[i][t];
#pragma unroll
                  for (int c = g * kSb; c < (g + 1) * kSb; ++c)
                    x[i][c] = fma(-l, s.psave[t][c], x[i][c]);
                }
            }
        }
      }
    }
    if (stop >= 0) break;
    // finished sub-panel columns to P (physical rows); shift the window
#pragma unroll
    for (int i = 0; i < kRpt; ++i) {
      if (lp[i] == kNone) continue;
      double* pc = P + tid + i * kThreads + (size_t)base * pr;
#pragma unroll
      for (int c = 0; c < kSb; ++c)
        if (c < sw) pc[c * pr] = x[i][c];
#pragma unroll
      for (int c = 0; c < kMaxNb - kSb; ++c) x[i][c] = x[i][c + kSb];
#pragma unroll
      for (int c = kMaxNb - kSb; c < kMaxNb; ++c) x[i][c] = 0.0;
    }
    base += kSb;
    if (base < w) {
      first_candidate(base, false);
      __syncthreads();
    }
  }
  // the window's remaining columns to P (physical rows)
#pragma unroll
  for (int i = 0; i < kRpt; ++i) {
    if (lp[i] == kNone) continue;
    double* pc = P + tid + i * kThreads;
#pragma unroll
    for (int c = 0; c < kMaxNb; ++c)
      if (base + c < w) pc[(size_t)(base + c) * pr] = x[i][c];
  }
  __syncthreads();
  // rows to their logical positions, in P and in the matrix
#pragma unroll
  for (int i = 0; i < kRpt; ++i) {
    if (lp[i] == kNone) continue;
    const double* pc = P + tid + i * kThreads;
#pragma unroll
    for (int c = 0; c < kMaxNb; ++c)
      if (c < w) x[i][c] = pc[c * pr];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kRpt; ++i) {
    if (lp[i] == kNone) continue;
    const int r = lp[i], phys = tid + i * kThreads;
#pragma unroll
    for (int c = 0; c < kMaxNb; ++c)
      if (c < w) {
        A[idx(b + r, b + c, lda)] = x[i][c];
        if (r != phys) P[r + c * pr] = x[i][c];
      }
    if (r != phys) {  // at most two rows per executed step move
      const int j = atomicAdd(&s.mv_count, 1);
      s.mv_dst[j] = (short)r;
      s.mv_src[j] = (short)phys;
    }
  }
  return stop;
}

// The panel's row permutation on every column outside it ([0, b) and
// [b + w, n)): four lanes per column gather all moved rows into registers
// (lane h takes the moves j == h mod 4), meet at a warp barrier, then store
// them at their destinations - no dependent swap chain.
__device__ __forceinline__ void permute_outside(double* A, int lda, int n, int b, int w,
                                                const Smem& s) {
  const int cnt = s.mv_count;
  if (cnt == 0) return;
  const int h = threadIdx.x & 3;
  const int total = n - w;
  for (int t0 = 0; t0 < total; t0 += kThreads / 4) {  // the same trip count for every lane
    const int t = t0 + ((int)threadIdx.x >> 2);
    const bool on = t < total;
    double* col = A + idx(b, on ? (t < b ? t : t + w) : 0, lda);
    double v[kMaxNb / 2];
#pragma unroll
    for (int q = 0; q < kMaxNb / 2; ++q) {
      const int j = 4 * q + h;
      if (on && j < cnt) v[q] = col[s.mv_src[j]];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < kMaxNb / 2; ++q) {
      const int j = 4 * q + h;
      if (on && j < cnt) col[s.mv_dst[j]] = v[q];
    }
  }
}

// Right of a panel that executed `kd` steps at [b, b + kd), its row
// permutation already applied: for the columns [c0, n), U12 = L11^{-1}
// A(b:b+kd, :) (written back) and A(b+kd:n, :) -= L21 U12, with L11 / L21 the
// shared panel P.  TERMS = 0: the product in FP64 (DMMA); TERMS = 2 / 3: the
// BF16 split product (3 / 6 products, FP32 accumulation), subtracted in FP64.
template <int TERMS>
__device__ __forceinline__ void trailing_update(double* A, int lda, int n, int b, int kd, int c0,
                                                const double* P, int pr, double* Bs) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  const int row0 = b + kd;
  const int M = n - row0, N = n - c0;
  const int kp = (kd + 3) & ~3;
  const double* L21 = P + kd;  // panel rows kd.. = matrix rows row0..
  for (int n0 = 0; n0 < N; n0 += kStageN) {
    const int ns = min(kStageN, N - n0);
    __syncthreads();  // Bs is free
    {
      double* bcol = Bs + tid * kLdb;
      if (tid < ns) {
        double* col = A + idx(0, c0 + n0 + tid, lda);
        double u[kMaxNb];
#pragma unroll
        for (int i = 0; i < kMaxNb; ++i) u[i] = i < kd ? col[b + i] : 0.0;
#pragma unroll
        for (int j = 0; j < kMaxNb - 1; ++j) {
          if (j >= kd) break;
          const double uj = u[j];
#pragma unroll
          for (int i = j + 1; i < kMaxNb; ++i)
            if (i < kd) u[i] = fma(-P[i + j * pr], uj, u[i]);
        }
#pragma unroll
        for (int i = 0; i < kMaxNb; ++i)
          if (i < kp) {
            if (i < kd) col[b + i] = u[i];
            bcol[i] = i < kd ? u[i] : 0.0;
          }
      } else {
        for (int i = 0; i < kp; ++i) bcol[i] = 0.0;
      }
    }
    __syncthreads();
    for (int h = 0; h * kTileN < ns; ++h) {
      const int nc = min(kTileN, ns - h * kTileN);
      const double* Bh = Bs + h * kTileN * kLdb;
      double* C = A + idx(row0, c0 + n0 + h * kTileN, lda);
      for (int m0 = 0; m0 < M; m0 += kTileM) {
        const int rb = m0 + wm * 32;
        if (rb >= M) continue;  // warp-uniform; no barrier inside this loop
        double cf[2][4][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              const int r = rb + mi * 16 + g + 8 * (v >> 1);
              const int c = wn * 32 + ni * 8 + 2 * t + (v & 1);
              cf[mi][ni][v] = (r < M && c < nc) ? C[idx(r, c, lda)] : 0.0;
            }
        double acc[2][4][4];
        if constexpr (TERMS == 0) {
#pragma unroll
          for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int v = 0; v < 4; ++v) acc[mi][ni][v] = 0.0;
          for (int k0 = 0; k0 < kp; k0 += 4) {
            const int kk = k0 + t;
            const bool kok = kk < kd;
            double a[2][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
              const int r = rb + mi * 16 + g;
              a[mi][0] = (kok && r < M) ? L21[r + kk * pr] : 0.0;
              a[mi][1] = (kok && r + 8 < M) ? L21[r + 8 + kk * pr] : 0.0;
            }
            double bf[4];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) bf[ni] = Bh[(wn * 32 + ni * 8 + g) * kLdb + kk];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
              for (int ni = 0; ni < 4; ++ni) mma_f64(acc[mi][ni], a[mi][0], a[mi][1], bf[ni]);
          }
        } else {
          // m16n8k16 fragments: A (row r, k) at r = g / g + 8 and k = 2t, 2t + 1,
          // 2t + 8, 2t + 9 of the 16-deep step; B (k, column) at the same k
          // for column g; C as the FP64 fragments above
          float facc[2][4][4];
#pragma unroll
          for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int v = 0; v < 4; ++v) facc[mi][ni][v] = 0.0f;
          for (int k0 = 0; k0 < kd; k0 += 16) {
            uint32_t af[TERMS][2][4], bfr[TERMS][4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
              for (int h = 0; h < 4; ++h) {  // register h: rows g (+8 for odd h), k pair
                const int r = rb + mi * 16 + g + 8 * (h & 1);
                const int kk = k0 + 2 * t + 8 * (h >> 1);
                __nv_bfloat16 lo[TERMS], hi[TERMS];
                split_pieces<TERMS>((r < M && kk < kd) ? L21[r + kk * pr] : 0.0, lo);
                split_pieces<TERMS>((r < M && kk + 1 < kd) ? L21[r + (kk + 1) * pr] : 0.0, hi);
#pragma unroll
                for (int q = 0; q < TERMS; ++q) af[q][mi][h] = pack_bf16(lo[q], hi[q]);
              }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const double* bc = Bh + (wn * 32 + ni * 8 + g) * kLdb;
                const int kk = k0 + 2 * t + 8 * h;
                __nv_bfloat16 lo[TERMS], hi[TERMS];
                split_pieces<TERMS>(kk < kd ? bc[kk] : 0.0, lo);
                split_pieces<TERMS>(kk + 1 < kd ? bc[kk + 1] : 0.0, hi);
#pragma unroll
                for (int q = 0; q < TERMS; ++q) bfr[q][ni][h] = pack_bf16(lo[q], hi[q]);
              }
#pragma unroll
            for (int d = 0; d < TERMS; ++d)
#pragma unroll
              for (int i = 0; i <= d; ++i)
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                  for (int ni = 0; ni < 4; ++ni) mma_bf16(facc[mi][ni], af[i][mi], bfr[d - i][ni]);
          }
#pragma unroll
          for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int v = 0; v < 4; ++v) acc[mi][ni][v] = (double)facc[mi][ni][v];
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              const int r = rb + mi * 16 + g + 8 * (v >> 1);
              const int c = wn * 32 + ni * 8 + 2 * t + (v & 1);
              if (r < M && c < nc) C[idx(r, c, lda)] = cf[mi][ni][v] - acc[mi][ni][v];
            }
      }
    }
  }
}

__device__ __forceinline__ bool better2(double va, int ca, int ra, double vb, int cb, int rb) {
  return va > vb || (va == vb && (ca < cb || (ca == cb && ra < rb)));
}

// 2-D argmax over the active block A(k:n, k:n): larger magnitude, then the
// smaller column, then the smaller row; NaN never wins.
__device__ __forceinline__ void active_argmax(const double* A, int lda, int n, int k, Smem& s,
                                              double& bv, int& br, int& bc, double& bs) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double v0 = -1.0, s0 = 0.0;  // best, runner-up (largest of the other magnitudes)
  int r0 = INT_MAX, c0 = INT_MAX;
  const int rows = n - k;
  for (int c = k; c < n; ++c)
    for (int r = tid; r < rows; r += kThreads) {
      const double v = fabs(A[idx(k + r, c, lda)]);
      if (v > v0) {  // (column, row) increase along this thread's scan
        s0 = fmax(s0, v0);
        v0 = v;
        r0 = k + r;
        c0 = c;
      } else {
        s0 = fmax(s0, v);
      }
    }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v0, off);
    const double os = __shfl_xor_sync(0xffffffffu, s0, off);
    const int orr = __shfl_xor_sync(0xffffffffu, r0, off);
    const int oc = __shfl_xor_sync(0xffffffffu, c0, off);
    if (better2(ov, oc, orr, v0, c0, r0)) {
      s0 = fmax(os, v0);
      v0 = ov;
      r0 = orr;
      c0 = oc;
    } else {
      s0 = fmax(s0, ov);
    }
  }
  __syncthreads();
  if (lane == 0) {
    s.fval[warp] = v0;
    s.fsec[warp] = s0;
    s.frow[warp] = r0;
    s.fcol[warp] = c0;
  }
  __syncthreads();
  bv = s.fval[0];
  bs = s.fsec[0];
  br = s.frow[0];
  bc = s.fcol[0];
  for (int q = 1; q < kWarps; ++q)
    if (better2(s.fval[q], s.fcol[q], s.frow[q], bv, bc, br)) {
      bs = fmax(s.fsec[q], bv);
      bv = s.fval[q];
      br = s.frow[q];
      bc = s.fcol[q];
    } else {
      bs = fmax(bs, s.fval[q]);
    }
}

template <int TERMS>
__device__ __forceinline__ void getrf_one(double* A, int n, int* ipiv, int* jpiv, int* info,
                                          int nb, double thr, double* P, int pr, double* Bs,
                                          Smem& s, unsigned long long* ties) {
  const int tid = threadIdx.x;
  const int lda = n;
  for (int i = tid; i < n; i += kThreads) ipiv[i] = jpiv[i] = i;
  if (tid == 0) *info = n;
  int b = 0;
  bool positioned = false;
  while (b < n) {
    const int w = min(nb, n - b), e = b + w;
    __syncthreads();  // P, Bs, the move list and the records are settled
    const int stop = panel_regs(A, n, lda, b, w, positioned, thr, P, pr, s, ipiv, ties);
    positioned = false;
    __syncthreads();  // panel written back, move list complete
    permute_outside(A, lda, n, b, w, s);
    if (stop < 0) {
      if (e < n) trailing_update<TERMS>(A, lda, n, b, w, e, P, pr, Bs);
      b = e;
      continue;
    }
    // column k has no acceptable pivot: bring the columns right of the panel
    // up to date for the executed steps, then search the whole active block
    const int k = b + stop;
    if (e < n && stop > 0) trailing_update<TERMS>(A, lda, n, b, stop, e, P, pr, Bs);
    __syncthreads();
    double bv, bs;
    int br, bc;
    active_argmax(A, lda, n, k, s, bv, br, bc, bs);
    if (tid == 0) note_tie(ties, k, bv > 0.0 ? bv : 0.0, bv > 0.0 ? bs : 0.0);
    if (!(bv > thr)) {
      if (tid == 0) *info = k;
      return;
    }
    if (tid == 0) {
      ipiv[k] = br;
      jpiv[k] = bc;
    }
    if (br != k)
      for (int c = tid; c < n; c += kThreads) {
        const double tmp = A[idx(k, c, lda)];
        A[idx(k, c, lda)] = A[idx(br, c, lda)];
        A[idx(br, c, lda)] = tmp;
      }
    __syncthreads();
    if (bc != k)
      for (int r = tid; r < n; r += kThreads) {
        const double tmp = A[idx(r, k, lda)];
        A[idx(r, k, lda)] = A[idx(r, bc, lda)];
        A[idx(r, bc, lda)] = tmp;
      }
    b = k;
    positioned = true;
  }
}

template <int TERMS>
__global__ void __launch_bounds__(kThreads, 1) batched_getrf_kernel(Params p) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ Smem s;
  double* P = dsm;
  double* Bs = dsm + (size_t)p.pr * kMaxNb;
  while (true) {
    __syncthreads();  // s.slot is free
    if (threadIdx.x == 0) s.slot = atomicAdd(p.queue, 1);
    __syncthreads();
    const int slot = s.slot;
    if (slot >= p.count) break;
    const int i = p.order[slot];
    const int n = p.ns[i];
    const int bk = bucket_of(n);  // selected without indexing the parameter array
    const int nb = bk == 0 ? p.nb_bucket[0] : bk == 1 ? p.nb_bucket[1] : bk == 2 ? p.nb_bucket[2]
                                                                                 : p.nb_bucket[3];
    getrf_one<TERMS>(p.base + p.offsets[i], n, p.ipiv + p.rec_offsets[i], p.jpiv + p.rec_offsets[i],
              p.info + i, nb, p.threshold, P, p.pr, Bs, s, p.ties);
  }
}

// One panel of the blocked LU (PanelParams, the same contract as
// panel_cluster_kernel) on ONE CTA, for panels of at most kMaxN rows and
// kMaxNb columns: the rows stay in registers and the pivot decisions,
// swaps (as relabelled row positions), scalings and rank-1 updates run with
// one CTA barrier per step and no cluster exchange (panel_regs, the batched
// kernel's panel).  Afterwards the composite row permutation is written as
// the swap lists the laswp kernel applies outside the panel.
__global__ void __launch_bounds__(kThreads, 1) panel_small_kernel(PanelParams p) {
  // every thread reads the same word before any barrier or state write
  if (p.gated && p.state->stop_k >= 0) return;
  extern __shared__ __align__(16) double dsm[];
  __shared__ Smem s;
  const int tid = threadIdx.x, lane = tid & 31;
  const int b = p.begin, w = p.end - p.begin;
  const int pr = panel_ld(p.m - b);
  if (tid == 0) {
    p.state->stop_k = -1;
    p.state->swap_count = 0;
    p.state->block_changed = 0;
  }
  const int stop = panel_regs(p.a, p.m, (int)p.lda, b, w, p.positioned != 0, p.threshold, dsm, pr,
                              s, p.ipiv, &p.state->ties_checked);
  __syncthreads();  // rows written back, move list complete
  for (int i = tid; i < w; i += kThreads) p.swap_block[i] = b + i;
  __syncthreads();
  const int cnt = s.mv_count;
  int changed = 0;
  for (int j0 = 0; j0 < cnt; j0 += kThreads) {  // whole warps: one atomic per warp
    const int j = j0 + tid;
    const bool on = j < cnt;
    const int dst = on ? s.mv_dst[j] : 0, src = on ? s.mv_src[j] : 0;
    if (on && dst < w) {
      p.swap_block[dst] = b + src;
      ++changed;
    }
    const bool below = on && dst >= w;
    const unsigned bal = __ballot_sync(0xffffffffu, below);
    if (bal) {
      int slot = 0;
      if (lane == 0) slot = atomicAdd(&p.state->swap_count, __popc(bal));
      slot = __shfl_sync(0xffffffffu, slot, 0) + __popc(bal & ((1u << lane) - 1u));
      if (below) {
        p.swap_extra[2 * slot + 0] = b + dst;
        p.swap_extra[2 * slot + 1] = b + src;
      }
    }
  }
  changed = __reduce_add_sync(0xffffffffu, changed);
  if (lane == 0 && changed) atomicAdd(&p.state->block_changed, changed);
  if (tid == 0 && stop >= 0) p.state->stop_k = b + stop;
}

size_t dynamic_smem(int max_n) {
  return ((size_t)panel_ld(std::max(max_n, 1)) * kMaxNb + (size_t)kStageN * kLdb) *
         sizeof(double);
}

// N(0,1) by the Box-Muller transform of two hashed uniforms (autotuner inputs).
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__global__ void fill_normal_kernel(double* x, long long len, uint64_t seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const uint64_t h1 = mix64(seed ^ mix64((uint64_t)i));
    const uint64_t h2 = mix64(h1);
    const double u1 = ((h1 >> 11) + 1) * (1.0 / 9007199254740992.0);
    const double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
    x[i] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}

}  // namespace batch
}  // namespace dp

// ---------------------------------------------------------------------------
// Host side: batch plans, launches, CUDA-graph replay, autotuner.

struct dp_batch {
  int device = 0;
  int count = 0;
  int max_n = 0;
  int sms = 0;
  long long total_elements = 0;
  long long total_records = 0;
  std::vector<int> n;
  std::vector<long long> offsets, rec_offsets;
  int* d_n = nullptr;
  long long* d_offsets = nullptr;
  long long* d_rec = nullptr;
  int* d_order = nullptr;
  int* d_queue = nullptr;
  dp_batch_options opt{};
  // captured graph and the arguments it was captured with
  cudaGraphExec_t exec = nullptr;
  const void* g_args[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace {

bool valid_batch_options(const dp_batch_options* o) {
  if (!(o->threshold >= 0.0) || std::isinf(o->threshold)) return false;
  if (!dp::valid_precision(o->precision)) return false;
  for (int i = 0; i < DP_BATCH_BUCKETS; ++i)
    if (o->nb_bucket[i] < 1 || o->nb_bucket[i] > DP_BATCH_MAX_NB) return false;
  return true;
}

int launch(dp_batch* bp, double* d_base, int* d_ipiv, int* d_jpiv, int* d_info, cudaStream_t st) {
  return dp::batch::launch_raw(bp->count, bp->max_n, bp->sms, bp->d_n, bp->d_offsets, bp->d_rec,
                               bp->d_order, bp->d_queue, d_base, d_ipiv, d_jpiv, d_info, bp->opt,
                               st);
}

bool aligned8(const void* p) { return ((uintptr_t)p & 7) == 0; }

}  // namespace

namespace dp {
namespace batch {

// The batched launch on caller-managed device arrays (the server's small-
// request path, which allocates from the stream-ordered pool): d_n, d_off,
// d_rec, d_order describe `count` matrices as in a dp_batch plan, d_queue is
// kQueueBytes of 8-byte aligned scratch (the work counter, then the launch's
// near-tie counters), cleared here before the launch.
int launch_raw(int count, int max_n, int sms, const int* d_n, const long long* d_off,
               const long long* d_rec, const int* d_order, int* d_queue, double* base, int* ipiv,
               int* jpiv, int* info, const dp_batch_options& opt, cudaStream_t st) {
  if (count <= 0) return DP_SUCCESS;
  if (max_n < 1 || max_n > DP_BATCH_MAX_N || !valid_batch_options(&opt)) return DP_INVALID_ARGUMENT;
  Params p;
  p.base = base;
  p.offsets = d_off;
  p.ns = d_n;
  p.rec_offsets = d_rec;
  p.order = d_order;
  p.count = count;
  p.queue = d_queue;
  p.ipiv = ipiv;
  p.jpiv = jpiv;
  p.info = info;
  p.ties = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(d_queue) + 8);
  p.threshold = opt.threshold;
  for (int i = 0; i < DP_BATCH_BUCKETS; ++i) p.nb_bucket[i] = opt.nb_bucket[i];
  p.pr = panel_ld(max_n);
  const size_t smem = dynamic_smem(max_n);
  const int terms = dp::mixed_terms(opt.precision);
  const void* fn = terms == 3   ? (const void*)batched_getrf_kernel<3>
                   : terms == 2 ? (const void*)batched_getrf_kernel<2>
                                : (const void*)batched_getrf_kernel<0>;
  if (!dp::ensure_smem(fn, smem)) return DP_CUDA_FAILURE;
  const int per_sm = dp::occupancy_once(fn, kThreads, smem);
  if (per_sm < 1) return DP_CUDA_FAILURE;
  const int grid = std::max(1, std::min(count, sms * per_sm));
  if (cudaMemsetAsync(d_queue, 0, kQueueBytes, st) != cudaSuccess) return DP_CUDA_FAILURE;
  dp::note_launch();
  void* args[] = {&p};
  if (cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, smem, st) != cudaSuccess)
    return DP_CUDA_FAILURE;
  return cudaGetLastError() == cudaSuccess ? DP_SUCCESS : DP_CUDA_FAILURE;
}

}  // namespace batch

void launch_fill_normal(double* x, long long len, unsigned long long seed, cudaStream_t st) {
  note_launch();
  batch::fill_normal_kernel<<<1184, 256, 0, st>>>(x, len, seed);
}

int panel_small_max_rows() { return batch::kMaxN; }
int panel_small_max_width() { return batch::kMaxNb; }

int launch_panel_small(const PanelParams& pp, cudaStream_t st) {
  const int rows = pp.m - pp.begin, w = pp.end - pp.begin;
  if (rows < 1 || rows > batch::kMaxN || w < 1 || w > batch::kMaxNb) return kInvalidArgument;
  const size_t smem = (size_t)batch::panel_ld(rows) * batch::kMaxNb * sizeof(double);
  if (!ensure_smem((const void*)batch::panel_small_kernel, smem)) return kCudaFailure;
  note_launch();
  batch::panel_small_kernel<<<1, batch::kThreads, smem, st>>>(pp);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

}  // namespace dp

namespace {

const int kBucketLo[DP_BATCH_BUCKETS] = {1, 64, 128, 256};
const int kBucketHi[DP_BATCH_BUCKETS] = {63, 127, 255, 512};

}  // namespace

extern "C" {

void dp_batch_options_init(dp_batch_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->threshold = 0.0;
  o->precision = DP_PRECISION_FP64;
  const int defaults[DP_BATCH_BUCKETS] = {16, 16, 32, 32};
  for (int i = 0; i < DP_BATCH_BUCKETS; ++i) o->nb_bucket[i] = defaults[i];
}

int dp_batch_create(dp_batch** out, int count, const int* n, const long long* offsets,
                    const dp_batch_options* opt) {
  if (!out) return DP_INVALID_ARGUMENT;
  *out = nullptr;
  if (count < 0 || (count > 0 && !n)) return DP_INVALID_ARGUMENT;
  dp_batch_options o;
  dp_batch_options_init(&o);
  if (opt) o = *opt;
  if (!valid_batch_options(&o)) return DP_INVALID_ARGUMENT;
  for (int i = 0; i < count; ++i)
    if (n[i] < 1 || n[i] > DP_BATCH_MAX_N || (offsets && offsets[i] < 0))
      return DP_INVALID_ARGUMENT;
  auto* bp = new (std::nothrow) dp_batch;
  if (!bp) return DP_ALLOCATION_FAILED;
  bp->opt = o;
  bp->count = count;
  bp->n.assign(n, n + count);
  bp->offsets.resize(count);
  bp->rec_offsets.resize(count);
  long long pos = 0, rec = 0;
  for (int i = 0; i < count; ++i) {
    bp->max_n = std::max(bp->max_n, n[i]);
    if (offsets) {
      bp->offsets[i] = offsets[i];
      pos = std::max(pos, offsets[i] + (long long)n[i] * n[i]);
    } else {
      bp->offsets[i] = pos;
      pos += ((long long)n[i] * n[i] + 3) & ~3LL;  // each matrix starts 32-byte aligned
    }
    bp->rec_offsets[i] = rec;
    rec += n[i];
  }
  bp->total_elements = pos;
  bp->total_records = rec;
  if (cudaGetDevice(&bp->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&bp->sms, cudaDevAttrMultiProcessorCount, bp->device) !=
          cudaSuccess) {
    delete bp;
    return DP_CUDA_FAILURE;
  }
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return bp->n[a] > bp->n[b]; });
  const size_t c = (size_t)std::max(count, 1);
  if (cudaMalloc(&bp->d_n, c * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&bp->d_offsets, c * sizeof(long long)) != cudaSuccess ||
      cudaMalloc(&bp->d_rec, c * sizeof(long long)) != cudaSuccess ||
      cudaMalloc(&bp->d_order, c * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&bp->d_queue, dp::batch::kQueueBytes) != cudaSuccess) {
    dp_batch_destroy(bp);
    return DP_ALLOCATION_FAILED;
  }
  if (count > 0 &&
      (cudaMemcpy(bp->d_n, bp->n.data(), count * sizeof(int), cudaMemcpyHostToDevice) !=
           cudaSuccess ||
       cudaMemcpy(bp->d_offsets, bp->offsets.data(), count * sizeof(long long),
                  cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(bp->d_rec, bp->rec_offsets.data(), count * sizeof(long long),
                  cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(bp->d_order, order.data(), count * sizeof(int), cudaMemcpyHostToDevice) !=
           cudaSuccess)) {
    dp_batch_destroy(bp);
    return DP_CUDA_FAILURE;
  }
  *out = bp;
  return DP_SUCCESS;
}

int dp_batch_layout(const dp_batch* bp, long long* offsets, long long* record_offsets,
                    long long* total_elements, long long* total_records) {
  if (!bp) return DP_INVALID_ARGUMENT;
  if (offsets) std::copy(bp->offsets.begin(), bp->offsets.end(), offsets);
  if (record_offsets) std::copy(bp->rec_offsets.begin(), bp->rec_offsets.end(), record_offsets);
  if (total_elements) *total_elements = bp->total_elements;
  if (total_records) *total_records = bp->total_records;
  return DP_SUCCESS;
}

int dp_batch_set_options(dp_batch* bp, const dp_batch_options* opt) {
  if (!bp || !opt || !valid_batch_options(opt)) return DP_INVALID_ARGUMENT;
  bp->opt = *opt;
  if (bp->exec) {  // the captured launch carries the old options
    cudaGraphExecDestroy(bp->exec);
    bp->exec = nullptr;
  }
  return DP_SUCCESS;
}

int dp_batch_getrf_async(dp_batch* bp, double* d_base, int* d_ipiv, int* d_jpiv, int* d_info,
                         void* stream) {
  if (!bp) return DP_INVALID_ARGUMENT;
  if (bp->count == 0) return DP_SUCCESS;
  if (!d_base || !d_ipiv || !d_jpiv || !d_info || !aligned8(d_base)) return DP_INVALID_ARGUMENT;
  return launch(bp, d_base, d_ipiv, d_jpiv, d_info, (cudaStream_t)stream);
}

int dp_batch_getrf_graph(dp_batch* bp, double* d_base, int* d_ipiv, int* d_jpiv, int* d_info,
                         void* stream) {
  if (!bp) return DP_INVALID_ARGUMENT;
  if (bp->count == 0) return DP_SUCCESS;
  if (!d_base || !d_ipiv || !d_jpiv || !d_info || !aligned8(d_base)) return DP_INVALID_ARGUMENT;
  const void* args[4] = {d_base, d_ipiv, d_jpiv, d_info};
  if (bp->exec && !std::equal(args, args + 4, bp->g_args)) {
    cudaGraphExecDestroy(bp->exec);
    bp->exec = nullptr;
  }
  if (!bp->exec) {
    cudaStream_t cap;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
      return DP_CUDA_FAILURE;
    cudaGraph_t graph = nullptr;
    int rc = DP_CUDA_FAILURE;
    if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const int lrc = launch(bp, d_base, d_ipiv, d_jpiv, d_info, cap);
      const cudaError_t ce = cudaStreamEndCapture(cap, &graph);
      if (lrc == DP_SUCCESS && ce == cudaSuccess &&
          cudaGraphInstantiate(&bp->exec, graph, 0) == cudaSuccess)
        rc = DP_SUCCESS;
      else
        rc = lrc != DP_SUCCESS ? lrc : DP_CUDA_FAILURE;
      if (graph) cudaGraphDestroy(graph);
    }
    cudaStreamDestroy(cap);
    if (rc != DP_SUCCESS) {
      cudaGetLastError();
      bp->exec = nullptr;
      return rc;
    }
    std::copy(args, args + 4, bp->g_args);
  }
  dp::note_launch();  // the graph holds one kernel (after the queue reset)
  return cudaGraphLaunch(bp->exec, (cudaStream_t)stream) == cudaSuccess ? DP_SUCCESS
                                                                        : DP_CUDA_FAILURE;
}

int dp_batch_last_report(dp_batch* bp, dp_getrf_report* out) {
  if (!bp || !out) return DP_INVALID_ARGUMENT;
  unsigned long long t[3] = {0, 0, 0};
  if (bp->count > 0 &&
      (cudaDeviceSynchronize() != cudaSuccess ||
       cudaMemcpy(t, reinterpret_cast<char*>(bp->d_queue) + 8, sizeof(t),
                  cudaMemcpyDeviceToHost) != cudaSuccess))
    return DP_CUDA_FAILURE;
  std::memset(out, 0, sizeof(*out));
  out->decisions = (long long)t[0];
  out->near_ties = (long long)t[1];
  std::memcpy(&out->max_closeness, &t[2], sizeof(double));
  out->info = bp->count;
  return DP_SUCCESS;
}

void dp_batch_destroy(dp_batch* bp) {
  if (!bp) return;
  if (bp->exec) cudaGraphExecDestroy(bp->exec);
  cudaFree(bp->d_n);
  cudaFree(bp->d_offsets);
  cudaFree(bp->d_rec);
  cudaFree(bp->d_order);
  cudaFree(bp->d_queue);
  delete bp;
}

// Autotuner: per size bucket, time every candidate panel width on seeded
// N(0,1) matrices whose orders spread log-uniformly over the bucket and keep
// the fastest.
int dp_batch_autotune(dp_batch_options* opt, int samples, unsigned long long seed,
                      void* stream) {
  if (!opt || samples < 1 || samples > 65536) return DP_INVALID_ARGUMENT;
  dp_batch_options base = *opt;
  if (!valid_batch_options(&base)) return DP_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  static const int kCand[] = {8, 16, 24, 32};
  int rc = DP_SUCCESS;
  for (int bk = 0; bk < DP_BATCH_BUCKETS && rc == DP_SUCCESS; ++bk) {
    const int lo = std::max(kBucketLo[bk], 16), hi = kBucketHi[bk];
    std::vector<int> ns(samples);
    for (int i = 0; i < samples; ++i) {
      const double f = samples > 1 ? (double)i / (samples - 1) : 0.5;
      const double v = std::exp(std::log((double)lo) + f * (std::log((double)hi) - std::log((double)lo)));
      ns[i] = std::min(std::max((int)std::lround(v), lo), hi);
    }
    dp_batch* bp = nullptr;
    rc = dp_batch_create(&bp, samples, ns.data(), nullptr, &base);
    if (rc != DP_SUCCESS) break;
    double *d_src = nullptr, *d_work = nullptr;
    int *d_ipiv = nullptr, *d_jpiv = nullptr, *d_info = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const size_t bytes = (size_t)bp->total_elements * sizeof(double);
    if (cudaMalloc(&d_src, bytes) != cudaSuccess || cudaMalloc(&d_work, bytes) != cudaSuccess ||
        cudaMalloc(&d_ipiv, bp->total_records * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_jpiv, bp->total_records * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_info, samples * sizeof(int)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      rc = DP_ALLOCATION_FAILED;
    } else {
      dp::note_launch();
      dp::batch::fill_normal_kernel<<<1184, 256, 0, st>>>(d_src, bp->total_elements,
                                                          seed + 0x1000003ull * bk);
      float best_ms = 1e30f;
      int best_nb = base.nb_bucket[bk];
      for (int nb : kCand) {
        dp_batch_options o = base;
        for (int q = 0; q < DP_BATCH_BUCKETS; ++q) o.nb_bucket[q] = nb;
        dp_batch_set_options(bp, &o);
        float ms_min = 1e30f;
        for (int rep = 0; rep < 3 && rc == DP_SUCCESS; ++rep) {
          if (cudaMemcpyAsync(d_work, d_src, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            rc = DP_CUDA_FAILURE;
            break;
          }
          cudaEventRecord(e0, st);
          rc = launch(bp, d_work, d_ipiv, d_jpiv, d_info, st);
          cudaEventRecord(e1, st);
          if (rc == DP_SUCCESS && cudaEventSynchronize(e1) != cudaSuccess) rc = DP_CUDA_FAILURE;
          float ms = 0.f;
          if (rc == DP_SUCCESS) cudaEventElapsedTime(&ms, e0, e1);
          ms_min = std::min(ms_min, ms);
        }
        if (rc != DP_SUCCESS) break;
        if (ms_min < best_ms) {
          best_ms = ms_min;
          best_nb = nb;
        }
      }
      if (rc == DP_SUCCESS) opt->nb_bucket[bk] = best_nb;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_src);
    cudaFree(d_work);
    cudaFree(d_ipiv);
    cudaFree(d_jpiv);
    cudaFree(d_info);
    dp_batch_destroy(bp);
  }
  return rc;
}

// Table file: one line per bucket, "<smallest n> <largest n> <nb>".
int dp_batch_tune_save(const char* path, const dp_batch_options* opt) {
  if (!path || !opt || !valid_batch_options(opt)) return DP_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "w");
  if (!f) return DP_INVALID_ARGUMENT;
  for (int i = 0; i < DP_BATCH_BUCKETS; ++i)
    std::fprintf(f, "%d %d %d\n", kBucketLo[i], kBucketHi[i], opt->nb_bucket[i]);
  return std::fclose(f) == 0 ? DP_SUCCESS : DP_INVALID_ARGUMENT;
}

int dp_batch_tune_load(const char* path, dp_batch_options* opt) {
  if (!path || !opt) return DP_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "r");
  if (!f) return DP_INVALID_ARGUMENT;
  dp_batch_options o = *opt;
  int rc = DP_SUCCESS;
  for (int i = 0; i < DP_BATCH_BUCKETS; ++i) {
    int lo, hi, nb;
    if (std::fscanf(f, "%d %d %d", &lo, &hi, &nb) != 3 || lo != kBucketLo[i] ||
        hi != kBucketHi[i] || nb < 1 || nb > DP_BATCH_MAX_NB) {
      rc = DP_INVALID_ARGUMENT;
      break;
    }
    o.nb_bucket[i] = nb;
  }
  std::fclose(f);
  if (rc == DP_SUCCESS) *opt = o;
  return rc;
}

}  // extern "C"
