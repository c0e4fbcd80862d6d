// Delayed Bunch-Kaufman LDL^T of a symmetric indefinite matrix on one B200:
// the blocked algorithm of delayed-bunch-kaufman/delayed_sytrf_blocked.cpp
// (and, with the same records, delayed_sytrf.cpp), lower triangle only.
//
// Per panel of up to nb columns (the reference's kBlockSize = 64, :23), one
// cooperative launch factors the columns one step at a time:
//   phase A  column k with this panel's update, A(k:n, k) - L_panel W(k, :)^T
//            (materialize_current_column, :75-88), written to `col`, and its
//            largest magnitude below the diagonal over the active rows with
//            the runner-up (cblas_idamax, :181-190);
//   phase B  when the diagonal fails criterion 1, the candidate row p over
//            [k, n) the same way (materialize_active_row, :90-106), to `row`,
//            and its largest off-diagonal magnitude over the active columns;
//   phase C  the decision of :192-235 (1x1 at k, 1x1 after swapping p to k,
//            2x2 (k, p) after swapping p to k + 1, or delay k to the end of
//            the active range), applied in one pass over the rows: the
//            symmetric swap of symmetric_swap_lower (:34-61) and the new L and
//            W = L D columns (:250-330) are fused, each element read and
//            written by one thread; the materialised columns after a swap are
//            the buffered ones re-indexed, so nothing is re-materialised.
// Phases are separated by a grid barrier (bounded wait); every CTA makes the
// same decision from the same buffered values.  The panel's trailing update
// (finish_panel, :126-139: dsyr2k of L and W) is the lower-triangle DMMA
// update C -= L W^T (launch_gemm_minus_lower).  W is kept transposed
// (WT, nb x n, column i = W's row i): its row swaps move 8 * pw contiguous
// bytes and the update reads it as a plain K x N operand.
#include <algorithm>
#include <climits>
#include <cstring>

#include <cuda_runtime.h>

#include "delayed_pivoting_b200.h"
#include "dp_device.cuh"
#include "dp_kernels.h"
#include "dp_stats.h"

namespace dp {
namespace bk {

constexpr double kAlpha = (1.0 + 4.1231056256176605498) / 8.0;  // (1 + sqrt 17) / 8
constexpr double kDetTol = 64.0 * 2.220446049250313080847e-16;  // 64 eps
constexpr double kUnit = 1.1102230246251565404e-16;               // u = 2^-53
constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kRowsPerWarp = 8;  // a warp: 8 rows x 4 interleaved groups of panel columns
constexpr int kRowsPerCta = kWarps * kRowsPerWarp;
constexpr int kMaxNb = 64;  // panel width limit (register-cached L entries)
constexpr int kPartsPerLane = 5;  // per-CTA partials one lane reduces: grid <= 160 CTAs
constexpr int kDefaultNb = 64;

// Largest magnitude, runner-up magnitude and the first index of the largest.
struct Top2 {
  double v, v2;
  int i, pad;
};

struct State {
  int k, e;             // next column to factor, end of the active range
  int status;           // kOk or kDeviceTimeout
  int pad;
  unsigned int bar[2];  // grid-barrier arrivals; launch parity selects one
  unsigned long long checked, near;  // decisions, order-sensitive decisions
  double closest;                    // largest closeness seen (1 = exact tie)
};

struct Params {
  double* a;
  long long lda;
  int n;
  double* wt;  // nb x n, leading dimension ldwt
  int ldwt, nb;
  double* col;  // materialised column, rows [k, n)
  double* row;  // materialised candidate row, columns [k, n)
  Top2* cpart;  // per-CTA column top-2
  double* rpart;  // per-CTA row maximum
  int* perm;
  int* piv;
  State* st;
};

enum Kind { kDelay = 0, kOne = 1, kOneSwap = 2, kTwo = 3, kBreak = 4 };

__device__ __forceinline__ double ld(const double* p) { return __ldcg(p); }

__device__ __forceinline__ void consider(Top2& t, double m, int i) {
  // rows arrive in increasing order per thread: an equal magnitude is a runner-up
  if (m > t.v) {
    t.v2 = t.v;
    t.v = m;
    t.i = i;
  } else if (m > t.v2) {
    t.v2 = m;
  }
}

// Top-2 of the union; equal magnitudes go to the smaller index (idamax's
// first occurrence) and count as a runner-up.  Commutative and associative,
// so every reduction order gives the same result.
__device__ __forceinline__ Top2 merge(Top2 a, Top2 b) {
  Top2 r;
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) {
    r.v = b.v;
    r.i = b.i;
    r.v2 = fmax(b.v2, a.v);
  } else {
    r.v = a.v;
    r.i = a.i;
    r.v2 = fmax(a.v2, b.v);
  }
  r.pad = 0;
  return r;
}

__device__ __forceinline__ Top2 warp_top2(Top2 t) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Top2 u;
    u.v = __shfl_xor_sync(~0u, t.v, o);
    u.v2 = __shfl_xor_sync(~0u, t.v2, o);
    u.i = __shfl_xor_sync(~0u, t.i, o);
    u.pad = 0;
    t = merge(t, u);
  }
  return t;
}

__device__ __forceinline__ double warp_max(double m) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(~0u, m, o));
  return m;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier over a monotonic arrival counter (all CTAs are co-resident:
// cooperative launch): the CTA's writes, ordered before thread 0 by the CTA
// barrier, are published by its release add; the acquire load that sees
// every arrival orders the CTA's later reads after all CTAs' writes.  The
// wait is bounded: after kSpinLimitNs the CTA records kDeviceTimeout and the
// caller returns.
__device__ __forceinline__ bool grid_barrier(unsigned int* ctr, unsigned int& target, int* status,
                                             int* s_ok) {
  target += gridDim.x;
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(ctr) : "memory");
    int ok = 1;
    unsigned long long t0 = 0;
    unsigned int it = 0;
    while (ld_acquire(ctr) < target) {
      if ((++it & 255u) == 0u) {
        const unsigned long long now = globaltimer_ns();
        if (t0 == 0) {
          t0 = now;
        } else if (now - t0 > kSpinLimitNs) {
          atomicExch(status, (int)kDeviceTimeout);
          ok = 0;
          break;
        }
      }
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Near-tie bookkeeping of one comparison x >= y of two magnitudes:
// closeness = min / max (1 = tie); `near` when closeness >= 1 - tol, and
// `closest` the largest closeness seen.  The division only runs when the
// ratio can raise `closest`.
__device__ __forceinline__ void tally(double x, double y, double tol, bool& near,
                                      double& closest) {
  x = fabs(x);
  y = fabs(y);
  const double hi = fmax(x, y), lo = fmin(x, y);
  if (!(hi > 0.0) || !isfinite(hi)) return;
  if (lo >= (1.0 - tol) * hi) near = true;
  if (lo > closest * hi) closest = lo / hi;
}

// stable_2x2 (delayed_sytrf_blocked.cpp:108-124); also returns |det| and the
// threshold it is compared with.
__device__ __forceinline__ bool stable_2x2(double a, double b, double c, double& det,
                                           double& thr) {
  det = thr = 0.0;
  const double s = fmax(fabs(a), fmax(fabs(b), fabs(c)));
  if (!(s > 0.0)) return false;
  const double as = a / s, bs = b / s, cs = c / s;
  det = fabs(as * cs - bs * bs);
  const double nrm = fmax(fabs(as) + fabs(bs), fabs(bs) + fabs(cs));
  thr = kDetTol * nrm * nrm;
  return det > thr;
}

// Rows of a panel are owned for the whole launch: slot s of CTA b holds the
// rows pb + (s G + b) 128 + [0, 128), a warp 8 of them; lane (q, r) of a warp
// serves row r of its 8 and keeps that row's panel columns j = q (mod 4) of
// L in registers (lr[t] = L(i, pb + q + 4 t)).  The panel products of phases
// A and B then read one global element per row; a row whose panel entries
// move (the two rows of a swap) reloads them after the step.
constexpr int kQ = kMaxNb / 4;  // cached L entries per lane and slot

__device__ __forceinline__ void swap_d(double* x, double* y) {
  const double t = ld(x);
  *x = ld(y);
  *y = t;
}

// The swap's far parts: rows x, y of the columns < c, and W's rows x, y
// (WT columns) over the pw panel columns.  A thread's first element of each
// is loaded before either is stored, so both loads share one round trip.
__device__ __forceinline__ void swap_far(double* a, long long lda, double* wt, long long ldwt,
                                         long long x, long long y, long long c, int pw,
                                         long long gt, long long gstride) {
  double u0 = 0.0, u1 = 0.0, w0 = 0.0, w1 = 0.0;
  const bool ha = gt < c, hw = gt < pw;
  if (ha) {
    u0 = ld(a + x + gt * lda);
    u1 = ld(a + y + gt * lda);
  }
  if (hw) {
    w0 = ld(wt + gt + x * ldwt);
    w1 = ld(wt + gt + y * ldwt);
  }
  if (ha) {
    a[x + gt * lda] = u1;
    a[y + gt * lda] = u0;
  }
  if (hw) {
    wt[gt + x * ldwt] = w1;
    wt[gt + y * ldwt] = w0;
  }
  for (long long i = gt + gstride; i < c; i += gstride) swap_d(a + x + i * lda, a + y + i * lda);
}

// sum over the cached panel columns of L(i, :) w, reduced over the row's 4 lanes.
__device__ __forceinline__ double row_dot(const double (&lr)[kQ], const double* s_w, int q) {
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int t = 0; t < kQ; t += 2) {
    s0 = fma(lr[t], s_w[q + 4 * t], s0);
    s1 = fma(lr[t + 1], s_w[q + 4 * t + 4], s1);
  }
  double s = s0 + s1;
  s += __shfl_xor_sync(~0u, s, 8);
  s += __shfl_xor_sync(~0u, s, 16);
  return s;
}

// lr <- L(i, pb + j) for the lane's columns j < pw (zero beyond).
__device__ __forceinline__ void load_row(double (&lr)[kQ], const double* a, long long lda,
                                         long long i, int pb, int pw, int q) {
#pragma unroll
  for (int t = 0; t < kQ; ++t) {
    const int j = q + 4 * t;
    lr[t] = j < pw ? ld(a + i + (long long)(pb + j) * lda) : 0.0;
  }
}

// lr's entry for panel column j <- v, in the lane that caches column j.
__device__ __forceinline__ void set_entry(double (&lr)[kQ], int q, int j, double v) {
  if ((j & 3) != q) return;
  const int tj = j >> 2;
#pragma unroll
  for (int t = 0; t < kQ; ++t)
    if (t == tj) lr[t] = v;
}

template <int RPT>
__global__ void __launch_bounds__(kThreads, 1) bk_panel_kernel(Params P, int parity) {
  __shared__ double s_w[kMaxNb];
  __shared__ Top2 s_t[kWarps];
  __shared__ double s_m[kWarps];
  __shared__ Top2 s_best;
  __shared__ double s_rowmax;
  __shared__ int s_ok;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = lane >> 3, r8 = lane & 7;
  const int G = gridDim.x;
  State* st = P.st;
  unsigned int* ctr = &st->bar[parity];
  if (blockIdx.x == 0 && tid == 0) st->bar[parity ^ 1] = 0u;  // the next launch's counter
  unsigned int target = 0;

  double* a = P.a;
  const long long lda = P.lda, ldwt = P.ldwt;
  const int n = P.n;
  int k = st->k, e = st->e;
  const int pb = k;
  int pw = 0;
  const long long gt = (long long)blockIdx.x * kThreads + tid;
  const long long gstride = (long long)G * kThreads;
  unsigned long long checked = 0, nnear = 0;
  double closest = 0.0;

  long long rowi[RPT];
  double lr[RPT][kQ], cv[RPT], rv[RPT], av[RPT], a1[RPT];
#pragma unroll
  for (int s = 0; s < RPT; ++s) {
    rowi[s] = pb + ((long long)s * G + blockIdx.x) * kRowsPerCta + warp * kRowsPerWarp + r8;
    cv[s] = rv[s] = av[s] = a1[s] = 0.0;
#pragma unroll
    for (int t = 0; t < kQ; ++t) lr[s][t] = 0.0;
  }
  long long rl0 = -1, rl1 = -1;  // rows whose cached entries are reloaded before phase A

  while (k < e && pw < P.nb) {
    // ---- phase A: column k of the panel-updated matrix, top-2 below the diagonal
#pragma unroll
    for (int s = 0; s < RPT; ++s) {
      const long long i = rowi[s];
      av[s] = (i >= k && i < n) ? ld(a + i + (long long)k * lda) : 0.0;
      if (i == rl0 || i == rl1) load_row(lr[s], a, lda, i, pb, pw, q);
    }
    for (int j = tid; j < kMaxNb; j += kThreads) s_w[j] = j < pw ? ld(P.wt + j + (long long)k * ldwt) : 0.0;
    __syncthreads();
    Top2 t{-1.0, -1.0, INT_MAX, 0};
#pragma unroll
    for (int s = 0; s < RPT; ++s) {
      const double v = av[s] - row_dot(lr[s], s_w, q);
      cv[s] = v;
      const long long i = rowi[s];
      if (q == 0 && i >= k && i < n) {
        P.col[i] = v;
        if (i > k && i < e) consider(t, fabs(v), (int)i);
      }
    }
    t = warp_top2(t);
    if (lane == 0) s_t[warp] = t;
    __syncthreads();
    if (warp == 0) {
      Top2 u = lane < kWarps ? s_t[lane] : Top2{-1.0, -1.0, INT_MAX, 0};
      u = warp_top2(u);
      if (lane == 0) P.cpart[blockIdx.x] = u;
    }
    if (!grid_barrier(ctr, target, &st->status, &s_ok)) return;

    // ---- phase B: the decision's inputs (every CTA reduces the same partials)
    const double dkk = ld(P.col + k);  // issued before the partials' loads: one round trip
    if (warp == 0) {
      // all of the lane's partials in flight at once (G <= 32 kPartsPerLane)
      Top2 c[kPartsPerLane];
#pragma unroll
      for (int r = 0; r < kPartsPerLane; ++r) {
        const int b = lane + 32 * r;
        c[r] = Top2{-1.0, -1.0, INT_MAX, 0};
        if (b < G) {
          c[r].v = ld(&P.cpart[b].v);
          c[r].v2 = ld(&P.cpart[b].v2);
          c[r].i = __ldcg(&P.cpart[b].i);
        }
      }
      Top2 u = c[0];
#pragma unroll
      for (int r = 1; r < kPartsPerLane; ++r) u = merge(u, c[r]);
      u = warp_top2(u);
      if (lane == 0) s_best = u;
    }
    __syncthreads();
    const Top2 best = s_best;
    int p = k;
    double colmax = 0.0;
    if (e - k > 1) {
      if (best.i != INT_MAX) {
        p = best.i;
        colmax = best.v;
      } else {  // every candidate NaN: none wins
        p = k + 1;
      }
    }
    const double akk = fabs(dkk);
    const bool any = fmax(akk, colmax) > 0.0;
    const bool c1 = any && akk >= kAlpha * colmax;
    double rowmax = 0.0, dpp = 0.0, d10 = 0.0, rowk = 0.0, rowk1 = 0.0, colk1 = 0.0;
    if (any && !c1) {
      // candidate row p over [k, n): symmetric A(p, i) - L(i, :) W(p, :)^T
      double sy[RPT];
#pragma unroll
      for (int s = 0; s < RPT; ++s) {
        const long long i = rowi[s];
        sy[s] = (i >= k && i < n) ? (i <= p ? ld(a + p + i * lda) : ld(a + i + (long long)p * lda))
                                  : 0.0;
        // A(i, k + 1): the old values a 2x2 step's swap relocates
        a1[s] = (i > k && i < n) ? ld(a + i + (long long)(k + 1) * lda) : 0.0;
      }
      for (int j = tid; j < kMaxNb; j += kThreads) s_w[j] = j < pw ? ld(P.wt + j + (long long)p * ldwt) : 0.0;
      __syncthreads();
      double m = 0.0;
#pragma unroll
      for (int s = 0; s < RPT; ++s) {
        const double v = sy[s] - row_dot(lr[s], s_w, q);
        rv[s] = v;
        const long long i = rowi[s];
        if (q == 0 && i >= k && i < n) {
          P.row[i] = v;
          if (i < e && i != p) m = fmax(m, fabs(v));
        }
      }
      m = warp_max(m);
      if (lane == 0) s_m[warp] = m;
      __syncthreads();
      if (warp == 0) {
        double u = lane < kWarps ? s_m[lane] : 0.0;
        u = warp_max(u);
        if (lane == 0) P.rpart[blockIdx.x] = u;
      }
      if (!grid_barrier(ctr, target, &st->status, &s_ok)) return;
      // every value the decision and phase C read from other rows, issued
      // with the partials' loads: one round trip
      dpp = ld(P.row + p);
      d10 = ld(P.col + p);
      rowk = ld(P.row + k);
      if (k + 1 < n) {
        rowk1 = ld(P.row + k + 1);
        colk1 = ld(P.col + k + 1);
      }
      if (warp == 0) {
        double c[kPartsPerLane];
#pragma unroll
        for (int r = 0; r < kPartsPerLane; ++r)
          c[r] = lane + 32 * r < G ? ld(P.rpart + lane + 32 * r) : 0.0;
        double u = c[0];
#pragma unroll
        for (int r = 1; r < kPartsPerLane; ++r) u = fmax(u, c[r]);
        u = warp_max(u);
        if (lane == 0) s_rowmax = u;
      }
      __syncthreads();
      rowmax = s_rowmax;
    }

    // ---- the decision (delayed_sytrf_blocked.cpp:192-235), identical in every CTA
    const double app = fabs(dpp);
    const double tol = 4.0 * (double)(k + 1) * kUnit;
    bool near = false;
    if (best.v2 >= 0.0) tally(best.v2, best.v, tol, near, closest);
    int kind = kDelay;
    double det = 0.0, thr = 0.0;
    if (any) {
      tally(akk, kAlpha * colmax, tol, near, closest);
      if (c1) {
        kind = kOne;
      } else {
        const double c2r = kAlpha * colmax * (colmax / rowmax);
        tally(akk, c2r, tol, near, closest);
        if (akk >= c2r) {
          kind = kOne;
        } else {
          tally(app, kAlpha * rowmax, tol, near, closest);
          if (app >= kAlpha * rowmax) {
            kind = kOneSwap;
          } else {
            const bool ok2 = stable_2x2(dkk, d10, dpp, det, thr);
            tally(det, thr, tol, near, closest);
            if (ok2) kind = pw + 2 > P.nb ? kBreak : kTwo;
          }
        }
      }
    }
    if (kind != kBreak) {  // counted by thread 0 of CTA 0; every thread tracks `closest`
      ++checked;
      if (near) ++nnear;
    }
    if (kind == kBreak) break;  // the 2x2 block starts the next panel (:245-248)

    // ---- phase C: the swap's far parts (columns < k) over all threads, the
    // new column(s) by the rows' owners from their own materialised values
    rl0 = rl1 = -1;
    if (kind == kDelay) {
      const int x = k, y = e - 1;
      if (x != y) {
        for (long long i = gt; i < n; i += gstride) {
          if (i < x) swap_d(a + x + i * lda, a + y + i * lda);
          else if (i == x) swap_d(a + x + (long long)x * lda, a + y + (long long)y * lda);
          else if (i < y) swap_d(a + i + (long long)x * lda, a + y + i * lda);
          else if (i > y) swap_d(a + i + (long long)x * lda, a + i + (long long)y * lda);
        }
        if (gt == gstride - 1) {
          const int t0 = P.perm[x];
          P.perm[x] = P.perm[y];
          P.perm[y] = t0;
        }
        for (long long j = gt; j < pw; j += gstride) swap_d(P.wt + j + x * ldwt, P.wt + j + y * ldwt);
        rl0 = x;
        rl1 = y;
      }
      e -= 1;
    } else if (kind == kOne) {
      const double d = dkk;
      if (gt == 0) P.piv[k] = 1;
#pragma unroll
      for (int s = 0; s < RPT; ++s) {
        const long long i = rowi[s];
        if (i < k || i >= n) continue;
        if (i == k) {
          if (q == 0) {
            a[i + i * lda] = d;
            P.wt[pw + i * ldwt] = d;
          }
        } else {
          const double l = cv[s] / d;
          if (q == 0) {
            a[i + (long long)k * lda] = l;
            P.wt[pw + i * ldwt] = cv[s];
          }
          set_entry(lr[s], q, pw, l);
        }
      }
      k += 1;
      pw += 1;
    } else if (kind == kOneSwap) {  // x = k, y = p: column k is rebuilt from `row`
      // owned rows first (the old A(i, k) the swap relocates is phase A's av),
      // then the swap's columns < k and W's rows
      const double d = dpp;
      if (gt == gstride - 1) {  // a thread with no column of the swap below (unless n > 512 G)
        P.piv[k] = 1;
        const int t0 = P.perm[k];
        P.perm[k] = P.perm[p];
        P.perm[p] = t0;
      }
#pragma unroll
      for (int s = 0; s < RPT; ++s) {
        const long long i = rowi[s];
        if (i < k || i >= n) continue;
        if (i == k) {
          if (q == 0) {
            a[p + (long long)p * lda] = av[s];
            a[k + (long long)k * lda] = d;
            P.wt[pw + i * ldwt] = d;
          }
        } else {
          const double b = i == p ? rowk : rv[s];
          const double l = b / d;
          if (q == 0) {
            if (i < p) a[p + i * lda] = av[s];
            else if (i > p) a[i + (long long)p * lda] = av[s];
            a[i + (long long)k * lda] = l;
            P.wt[pw + i * ldwt] = b;
          }
          set_entry(lr[s], q, pw, l);
        }
      }
      swap_far(a, lda, P.wt, ldwt, k, p, k, pw, gt, gstride);
      rl0 = p;
      k += 1;
      pw += 1;
    } else {  // kTwo: x = k + 1, y = p; columns k, k + 1 from `col`, `row`
      const bool sw = p != k + 1;
      const double d00 = dkk, d11 = dpp;
      const double sc = fmax(fabs(d00), fmax(fabs(d10), fabs(d11)));
      const double s00 = d00 / sc, s10 = d10 / sc, s11 = d11 / sc;
      const double inv = 1.0 / (sc * (s00 * s11 - s10 * s10));
      const long long k1 = k + 1;
      if (gt == gstride - 1) {
        P.piv[k] = 2;
        P.piv[k1] = 0;
        if (sw) {
          const int t0 = P.perm[k1];
          P.perm[k1] = P.perm[p];
          P.perm[p] = t0;
        }
      }
#pragma unroll
      for (int s = 0; s < RPT; ++s) {
        const long long i = rowi[s];
        if (i < k || i >= n) continue;
        if (i == k) {
          if (q == 0) {
            a[k + (long long)k * lda] = d00;
            a[k1 + (long long)k * lda] = d10;
            P.wt[pw + i * ldwt] = d00;
            P.wt[pw + 1 + i * ldwt] = d10;
          }
        } else if (i == k1) {
          if (q == 0) {
            if (sw) a[p + (long long)p * lda] = a1[s];  // old A(k + 1, k + 1)
            a[k1 + k1 * lda] = d11;
            P.wt[pw + i * ldwt] = d10;
            P.wt[pw + 1 + i * ldwt] = d11;
          }
        } else {
          const bool moved = sw && i == p;
          const double b0 = moved ? colk1 : cv[s], b1 = moved ? rowk1 : rv[s];
          const double l0 = (s11 * b0 - s10 * b1) * inv;
          const double l1 = (s00 * b1 - s10 * b0) * inv;
          if (q == 0) {
            if (sw) {  // old A(i, k + 1), loaded with the row
              if (i < p) a[p + i * lda] = a1[s];
              else if (i > p) a[i + (long long)p * lda] = a1[s];
            }
            a[i + (long long)k * lda] = l0;
            a[i + k1 * lda] = l1;
            P.wt[pw + i * ldwt] = b0;
            P.wt[pw + 1 + i * ldwt] = b1;
          }
          set_entry(lr[s], q, pw, l0);
          set_entry(lr[s], q, pw + 1, l1);
        }
      }
      if (sw) {
        swap_far(a, lda, P.wt, ldwt, k1, p, k, pw, gt, gstride);
        rl0 = p;
      }
      k += 2;
      pw += 2;
    }
    if (k < e && pw < P.nb) {
      if (!grid_barrier(ctr, target, &st->status, &s_ok)) return;
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    st->k = k;
    st->e = e;
    st->checked += checked;
    st->near += nnear;
    st->closest = fmax(st->closest, closest);
  }
}

// Kernel instance for RPT rows per lane (slots), nullptr beyond kMaxSlots.
constexpr int kMaxSlots = 4;
const void* panel_kernel_for(int slots) {
  switch (slots) {
    case 1: return (const void*)bk_panel_kernel<1>;
    case 2: return (const void*)bk_panel_kernel<2>;
    case 3:
    case 4: return (const void*)bk_panel_kernel<4>;
    default: return nullptr;
  }
}


__global__ void bk_init_kernel(int n, int* perm, int* piv, State* st) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    perm[i] = (int)i;
    piv[i] = 0;
  }
  if (i == 0) {
    st->k = 0;
    st->e = n;
    st->status = kOk;
    st->bar[0] = st->bar[1] = 0u;
    st->checked = st->near = 0ull;
    st->closest = 0.0;
  }
}

}  // namespace bk

namespace {

thread_local dp_getrf_report g_bk_report = {0, 0, 0.0, -1, {0, 0, 0}};

// CTAs of a cooperative launch of the panel kernel: one per SM at most.
int panel_ctas_max() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  int sms = 0, coop = 0, per = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bk::bk_panel_kernel<4>,
                                                              bk::kThreads, 0) != cudaSuccess)
    return 0;
  return per > 0 ? sms : 0;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Mean panel columns in the products of a launch that factored w columns.
double pw_avg_dot(int w) { return w > 0 ? 0.5 * (w - 1) : 0.0; }

}  // namespace

// perm / piv_size: host arrays of n entries.  Synchronises `s`.
int sytrf_device(int n, double* d_a, int lda, int* perm, int* piv_size, int* info, cudaStream_t s,
                 int nb, int grid) {
  g_bk_report = dp_getrf_report{0, 0, 0.0, -1, {0, 0, 0}};
  if (info) *info = -1;
  if (n < 0 || lda < std::max(1, n) || !info || (n > 0 && (!d_a || !perm || !piv_size)))
    return kInvalidArgument;
  if (nb == 0) nb = bk::kDefaultNb;
  if (nb < 2 || nb > bk::kMaxNb || grid < 0) return kInvalidArgument;
  if (n == 0) {
    *info = 0;
    g_bk_report.info = 0;
    return kOk;
  }
  const int gmax = panel_ctas_max();
  if (gmax <= 0) return kCudaFailure;
  int G = grid > 0 ? grid : (n + bk::kRowsPerCta - 1) / bk::kRowsPerCta;
  G = std::max(1, std::min({G, gmax, 32 * bk::kPartsPerLane}));
  // each lane caches the panel rows of at most kMaxSlots slots of 128 rows per CTA
  if ((long long)n > (long long)G * bk::kRowsPerCta * bk::kMaxSlots) return kInvalidArgument;

  const size_t b_wt = align256((size_t)nb * n * sizeof(double));
  const size_t b_vec = align256((size_t)n * sizeof(double));
  const size_t b_cp = align256((size_t)G * sizeof(bk::Top2));
  const size_t b_rp = align256((size_t)G * sizeof(double));
  const size_t b_int = align256((size_t)n * sizeof(int));
  const size_t total = b_wt + 2 * b_vec + b_cp + b_rp + 2 * b_int + align256(sizeof(bk::State));
  char* ws = nullptr;
  if (cudaMallocAsync((void**)&ws, total, s) != cudaSuccess) return kAllocationFailed;
  bk::State hs;  // the panel kernel's state, read after each launch (a few bytes)
  bk::State* h = &hs;
  bk::Params P;
  char* c = ws;
  P.wt = (double*)c;
  c += b_wt;
  P.col = (double*)c;
  c += b_vec;
  P.row = (double*)c;
  c += b_vec;
  P.cpart = (bk::Top2*)c;
  c += b_cp;
  P.rpart = (double*)c;
  c += b_rp;
  P.perm = (int*)c;
  c += b_int;
  P.piv = (int*)c;
  c += b_int;
  P.st = (bk::State*)c;
  P.a = d_a;
  P.lda = lda;
  P.n = n;
  P.ldwt = nb;
  P.nb = nb;

  int status = kOk;
  // dp_stats families: panel launches, the lower DMMA updates, the record init
  Recorder rec(s);
  rec.begin(DP_KFAM_OTHER);
  note_launch();
  bk::bk_init_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, P.perm, P.piv, P.st);
  rec.end(0.0, 8.0 * n + sizeof(bk::State), 1);
  if (cudaGetLastError() != cudaSuccess) status = kCudaFailure;
  int pb = 0, e = n, parity = 0;
  while (status == kOk) {
    void* args[] = {(void*)&P, (void*)&parity};
    note_launch();
    rec.begin(DP_KFAM_PANEL);
    const long long per_slot = (long long)G * bk::kRowsPerCta;
    const int slots = (int)((n - pb + per_slot - 1) / per_slot);
    if (cudaLaunchCooperativeKernel(bk::panel_kernel_for(slots), dim3(G), dim3(bk::kThreads), args,
                                    0, s) != cudaSuccess ||
        cudaMemcpyAsync(h, P.st, sizeof(bk::State), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      status = kCudaFailure;
      break;
    }
    {
      // algorithmic traffic of the launch: per factored column the column and
      // row reads and the L and W column writes over the rows below pb
      const double w = (double)(h->k - pb), rows = (double)(n - pb);
      rec.end(4.0 * w * rows * pw_avg_dot(h->k - pb), 32.0 * w * rows, 1);
    }
    if (h->status != kOk) {
      status = h->status;
      break;
    }
    const int k = h->k;
    if (k == pb && h->e == e) {  // every launch factors or delays at least one column
      status = kLibraryFailure;
      break;
    }
    e = h->e;
    // finish_panel: the trailing block [k, n), delayed suffix included
    if (k > pb && k < n) {
      const double t = (double)(n - k), w = (double)(k - pb);
      rec.begin(DP_KFAM_GEMM);
      launch_gemm_minus_lower(n - k, k - pb, d_a + k + (long long)pb * lda, lda,
                              P.wt + (long long)k * nb, nb, d_a + k + (long long)k * lda, lda, s);
      // lower triangle: t (t + 1) w flops; C read and written once, L and W read
      rec.end(t * (t + 1.0) * w, 8.0 * t * (t + 1.0) + 16.0 * t * w, 1);
    }
    pb = k;
    parity ^= 1;
    if (k >= e) break;
  }
  if (status == kOk &&
      (cudaMemcpyAsync(perm, P.perm, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaMemcpyAsync(piv_size, P.piv, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, s) !=
           cudaSuccess))
    status = kCudaFailure;
  cudaFreeAsync(ws, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && status == kOk) status = kCudaFailure;
  rec.flush(status == kOk);
  if (status == kOk) {
    *info = e;
    g_bk_report.decisions = (long long)h->checked;
    g_bk_report.near_ties = (long long)h->near;
    g_bk_report.max_closeness = h->closest;
    g_bk_report.info = e;
  }
  return status;
}

}  // namespace dp

extern "C" {

void dp_sytrf_options_init(dp_sytrf_options* opt) {
  if (opt) std::memset(opt, 0, sizeof(*opt));
}

int dp_sytrf_device_ex(int n, double* d_a, int lda, int* perm, int* piv_size, int* info,
                       const dp_sytrf_options* opt, void* stream) {
  return dp::sytrf_device(n, d_a, lda, perm, piv_size, info, static_cast<cudaStream_t>(stream),
                          opt ? opt->nb : 0, opt ? opt->grid : 0);
}

int dp_sytrf_device(int n, double* d_a, int lda, int* perm, int* piv_size, int* info,
                    void* stream) {
  return dp_sytrf_device_ex(n, d_a, lda, perm, piv_size, info, nullptr, stream);
}

int dp_sytrf_host(int n, double* a, int lda, int* perm, int* piv_size, int* info) {
  if (info) *info = -1;
  if (n < 0 || lda < std::max(1, n) || !info || (n > 0 && (!a || !perm || !piv_size)))
    return dp::kInvalidArgument;
  if (n == 0) return dp_sytrf_device(0, nullptr, lda, perm, piv_size, info, nullptr);
  const size_t bytes = (size_t)lda * n * sizeof(double);
  double* d = nullptr;
  if (cudaMalloc((void**)&d, bytes) != cudaSuccess) return dp::kAllocationFailed;
  int status = cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice) == cudaSuccess
                   ? dp_sytrf_device(n, d, lda, perm, piv_size, info, nullptr)
                   : (int)dp::kCudaFailure;
  if (status == dp::kOk && cudaMemcpy(a, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
    status = dp::kCudaFailure;
    *info = -1;
  }
  cudaFree(d);
  return status;
}

int dp_sytrf_last_report(dp_getrf_report* report) {
  if (!report) return dp::kInvalidArgument;
  *report = dp::g_bk_report;
  return dp::kOk;
}

}  // extern "C"

// C++ drop-ins for the reference's CPU entry points
// (delayed-bunch-kaufman/delayed_sytrf.hpp:15, delayed_sytrf_blocked.hpp:15):
// host memory in and out, the factorisation on the current GPU; info = -1 on
// any failure, as the reference does for invalid arguments.
void delayed_sytrf_blocked(int n, double* a, int lda, int* perm, int* piv_size, int& info) {
  int i = -1;
  if (dp_sytrf_host(n, a, lda, perm, piv_size, &i) != dp::kOk) i = -1;
  info = i;
}

void delayed_sytrf(int n, double* a, int lda, int* perm, int* piv_size, int& info) {
  delayed_sytrf_blocked(n, a, lda, perm, piv_size, info);
}
