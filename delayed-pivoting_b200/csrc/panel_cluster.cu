// Panel factorisation of the delayed-pivoting LU inside one thread-block
// cluster (up to 16 CTAs on 16 SMs of one GPC).
//
// Same semantics as panel_factor_kernel (delayed_lu/delayed_dgetrf.cpp:164-240:
// column partial-pivot search with first-index ties and NaN never winning,
// acceptance |alpha| > threshold, row swap inside the panel, scaling by the
// reciprocal pivot, rank-1 update of the remaining panel columns, stop at the
// first column without an acceptable pivot), but every per-column exchange
// goes through distributed shared memory instead of L2:
//   1. each CTA finds its local candidate (fused into the previous update);
//   2. it pushes (value, row), its candidate row and - on the owner of row
//      k - row k into every CTA's shared memory (st.shared::cluster);
//   3. one hardware cluster barrier (arrive.release / wait.acquire);
//   4. every CTA picks the same winner from the C candidates, finds the pivot
//      row and row k already in its own shared memory, and swaps, scales and
//      updates its own rows.
// One barrier and no round trip per column.  The rank-1 updates are confined
// to sub-panels of kSub columns: every CTA keeps the sub-panel's pivot rows as
// they were pushed, and at the sub-panel's end solves them for the remaining
// panel columns (U12 = L11^{-1} A12, identical in every CTA) and applies one
// rank-kSub update to its rows - the shared-memory traffic of the update drops
// from (w - s) columns per step to kSub.  Push buffers are indexed by
// step parity: a buffer written at step s + 2 is written after the barrier
// of step s + 1, which a reader of step s passes only after finishing step
// s.  No spin-waits: the only waits are the hardware barrier.
#include <cooperative_groups.h>

#include "dp_device.cuh"
#include "dp_kernels.h"

namespace cg = cooperative_groups;

namespace dp {

namespace {

constexpr int kThreads = 256;
constexpr int kSub = 8;  // sub-panel width

struct __align__(16) CandSlot {
  double val;
  int row;     // global row, -1 when the CTA has no candidate
  int pad;
  double inv;  // reciprocal of the candidate's entry in the current column
  double pad2;
};

struct __align__(16) LocalBest {
  double val;
  int row;  // local row, -1 when none
  int pad;
};

// Best (largest magnitude, then smallest row) over the warp's lanes, every
// lane getting the result.  Magnitudes are >= 0 and a missing candidate
// offers (0, INT_MAX), so the bit patterns order like the values: max of the
// high word, of the low word among its holders, then min row - three warp
// reductions instead of five shuffle rounds.
__device__ __forceinline__ void warp_best(double v, int row, double& bv, int& brow) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(u >> 32), lo = (unsigned)u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const int key = (hi == mhi && lo == mlo) ? row : 0x7fffffff;
  brow = __reduce_min_sync(0xffffffffu, key);
  bv = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

__device__ __forceinline__ LocalBest warp_lb(LocalBest v) {
  double bv;
  int br;
  warp_best(v.row >= 0 ? v.val : 0.0, v.row >= 0 ? v.row : 0x7fffffff, bv, br);
  return LocalBest{br == 0x7fffffff ? 0.0 : bv, br == 0x7fffffff ? -1 : br, 0};
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 1) panel_cluster_kernel(PanelParams p) {
  // Every CTA reads the same word before any barrier or state write (a stop
  // is recorded only by an earlier kernel), so all of them leave together.
  if (p.gated && p.state->stop_k >= 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int w = p.end - p.begin;
  const int W1 = w + 1;  // row values + source-row index
  const int R = p.rows_per_cta;
  const int RP = R | 1;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int nwarps = (int)(blockDim.x >> 5);
  const long long row0 = (long long)p.begin + (long long)rank * R;
  const int rows_here = (int)max(0LL, min((long long)R, (long long)p.m - row0));

  // Shared layout: panel slice; candidate slots [2 parity][16]; candidate
  // rows pushed by every CTA [2 parity][16][w + 1]; row k [2 parity][w + 1];
  // source row of each local row.
  double* sm = reinterpret_cast<double*>(smem_raw);  // [w][RP]
  const size_t sm_elems = ((size_t)w * RP + 1) & ~(size_t)1;  // next region 16-byte aligned
  CandSlot* cands = reinterpret_cast<CandSlot*>(sm + sm_elems);
  double* stc = reinterpret_cast<double*>(cands + 32);  // candidate rows
  double* stk = stc + (size_t)2 * 16 * W1;              // row k
  double* psave = stk + (size_t)2 * W1;  // [kSub][W1]: the sub-panel's pivot rows
  int* orig = reinterpret_cast<int*>(psave + (size_t)kSub * W1);
  __shared__ LocalBest red[kThreads / 32];

  for (int c = 0; c < w; ++c) {
    const double* src = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += blockDim.x) sm[(size_t)c * RP + r] = src[r];
  }
  for (int r = tid; r < rows_here; r += blockDim.x) orig[r] = (int)(row0 + r);
  if (rank == 0 && tid == 0) {
    p.state->stop_k = -1;
    p.state->swap_count = 0;
    p.state->block_changed = 0;
  }
  __syncthreads();

  LocalBest mine{0.0, -1, 0};
  {
    const int kl0 = (int)((long long)p.begin - row0);
    for (int r = max(0, kl0) + tid; r < rows_here; r += blockDim.x) {
      const double v = fabs(sm[r]);
      if (v > mine.val) {
        mine.val = v;
        mine.row = r;
      }
    }
  }

  // End of a sub-panel that executed kd steps at [base, base + kd): solve its
  // pivot rows for the columns [send, w) and update the rows below; then
  // the candidate of column send (unless the panel stopped).
  auto sub_panel_end = [&](int kd, int base, int send) {
    __syncthreads();  // psave complete, this CTA's rows updated
    if (kd > 0) {
      for (int c = send + tid; c < w; c += blockDim.x)
        for (int j = 1; j < kd; ++j) {
          double u = psave[(size_t)j * W1 + c];
          for (int t = 0; t < j; ++t)
            u -= psave[(size_t)j * W1 + base + t] * psave[(size_t)t * W1 + c];
          psave[(size_t)j * W1 + c] = u;
        }
      __syncthreads();
      const long long first = (long long)p.begin + base;  // global row of the first pivot
      for (int r = tid; r < rows_here; r += blockDim.x) {
        const long long g = row0 + r;
        double* __restrict__ row = sm + r;
        if (g < first) continue;
        if (g < first + kd) {
          const double* u = psave + (size_t)(g - first) * W1;
          for (int c = send; c < w; ++c) row[(size_t)c * RP] = u[c];
          continue;
        }
        double l[kSub];
#pragma unroll
        for (int t = 0; t < kSub; ++t) l[t] = t < kd ? row[(size_t)(base + t) * RP] : 0.0;
        for (int c = send; c < w; ++c) {
          double x = row[(size_t)c * RP];
#pragma unroll
          for (int t = 0; t < kSub; ++t)
            if (t < kd) x = fma(-l[t], psave[(size_t)t * W1 + c], x);
          row[(size_t)c * RP] = x;
        }
      }
    }
    __syncthreads();
    mine = LocalBest{0.0, -1, 0};
    if (send < w) {
      const long long last = (long long)p.begin + base + kd - 1;  // last pivot row
      for (int r = tid; r < rows_here; r += blockDim.x) {
        if (row0 + r <= last) continue;
        const double v = fabs(sm[(size_t)send * RP + r]);
        if (v > mine.val) {
          mine.val = v;
          mine.row = r;
        }
      }
    }
  };

  for (int s = 0; s < w; ++s) {
    const long long k = (long long)p.begin + s;
    const int par = s & 1;
    const bool positioned = (s == 0) && p.positioned;
    const int kl = (int)(k - row0);
    const bool own_k = kl >= 0 && kl < rows_here;

    // 1. CTA candidate (every thread reduces the per-warp results itself).
    if (positioned) {
      mine = LocalBest{0.0, -1, 0};
      if (own_k && tid == 0) mine = LocalBest{__longlong_as_double(0x7ff0000000000000ll), kl, 0};
    }
    mine = warp_lb(mine);
    if (lane == 0) red[warp] = mine;
    __syncthreads();
    const LocalBest cb = warp_lb(lane < nwarps ? red[lane] : LocalBest{0.0, -1, 0});

    // 2. Push (value, row), the candidate row and row k into every CTA.
    {
      double* my_stc = stc + ((size_t)par * 16 + rank) * W1;
      double* my_stk = stk + (size_t)par * W1;
      // warp w pushes to CTAs w, w + nwarps, ...; its lanes walk the row
      if (cb.row >= 0 || own_k) {
        for (int dest = warp; dest < C; dest += nwarps)
          for (int j = lane; j < W1; j += 32) {
            if (cb.row >= 0) {
              const double v = j < w ? sm[(size_t)j * RP + cb.row] : (double)orig[cb.row];
              *cluster.map_shared_rank(my_stc + j, dest) = v;
            }
            if (own_k) {
              const double v = j < w ? sm[(size_t)j * RP + kl] : (double)orig[kl];
              *cluster.map_shared_rank(my_stk + j, dest) = v;
            }
          }
      }
      if (tid < C) {
        CandSlot cs;
        cs.val = cb.row >= 0 ? cb.val : 0.0;
        cs.row = cb.row >= 0 ? (int)(row0 + cb.row) : -1;
        cs.pad = 0;
        cs.inv = cb.row >= 0 ? 1.0 / sm[(size_t)s * RP + cb.row] : 0.0;
        cs.pad2 = 0.0;
        *cluster.map_shared_rank(cands + par * 16 + rank, tid) = cs;
      }
    }
    cluster.sync();

    // 3. Same decision everywhere; the pivot row and row k are local now.
    CandSlot win{0.0, -1, 0, 0.0, 0.0};
    {
      const CandSlot c = lane < C ? cands[par * 16 + lane] : CandSlot{0.0, -1, 0, 0.0, 0.0};
      double bv;
      int brow;
      warp_best(c.row >= 0 ? c.val : 0.0, c.row >= 0 ? c.row : 0x7fffffff, bv, brow);
      if (brow != 0x7fffffff) {
        // the slot holding the winner (global rows are unique)
        const int src = __ffs(__ballot_sync(0xffffffffu, c.row == brow && lane < C)) - 1;
        win.val = bv;
        win.row = brow;
        win.inv = __shfl_sync(0xffffffffu, c.inv, max(src, 0));
      }
    }
    const bool stop = !positioned && !(win.row >= 0 && win.val > p.threshold);
    if (stop) {
      if (rank == 0 && tid == 0) p.state->stop_k = (int)k;
      // the columns right of the sub-panel take its executed steps
      const int base = (s / kSub) * kSub, send = min(base + kSub, w);
      if (send < w) sub_panel_end(s - base, base, send);
      break;
    }
    const long long prow_g = win.row;
    const int owner_p = (int)((prow_g - p.begin) / R);
    const double* __restrict__ pr = stc + ((size_t)par * 16 + owner_p) * W1;
    const double* __restrict__ kr = stk + (size_t)par * W1;
    const int pl = (int)(prow_g - row0);
    const bool swap_p = pl >= 0 && pl < rows_here && prow_g != k;
    if (rank == 0 && tid == 0 && !positioned) p.ipiv[k] = (int)prow_g;
    const int base = (s / kSub) * kSub, send = min(base + kSub, w);
    for (int j = tid; j < W1; j += blockDim.x) psave[(size_t)(s - base) * W1 + j] = pr[j];

    // 4. Swap, scale, update own rows; next column's candidate on the way.
    const double inv = win.inv;
    mine = LocalBest{0.0, -1, 0};
    for (int r = max(0, kl) + tid; r < rows_here; r += blockDim.x) {
      double* __restrict__ row = sm + r;
      if (r == kl) {
        for (int j = 0; j < w; ++j) row[(size_t)j * RP] = pr[j];
        orig[r] = (int)pr[w];
        continue;
      }
      if (swap_p && r == pl) {
        for (int j = 0; j < w; ++j) row[(size_t)j * RP] = kr[j];
        orig[r] = (int)kr[w];
      }
      const double l = row[(size_t)s * RP] * inv;
      row[(size_t)s * RP] = l;
      if (s + 1 < send) {  // columns past the sub-panel wait for its rank-kSub update
        const double v = row[(size_t)(s + 1) * RP] - l * pr[s + 1];
        row[(size_t)(s + 1) * RP] = v;
        const double av = fabs(v);
        if (av > mine.val) {
          mine.val = av;
          mine.row = r;
        }
        for (int j = s + 2; j < send; ++j) row[(size_t)j * RP] -= l * pr[j];
      }
    }
    if (s + 1 == send && send < w) sub_panel_end(s + 1 - base, base, send);
  }
  // Rows were swapped and updated by other threads than those writing them
  // back, and no CTA may exit while a peer could still push into it.
  cluster.sync();

  for (int c = 0; c < w; ++c) {
    double* dst = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += blockDim.x) dst[r] = sm[(size_t)c * RP + r];
  }
  for (int r = tid; r < rows_here; r += blockDim.x) {
    const long long g = row0 + r;
    const int src = orig[r];
    if (g < p.end) {
      p.swap_block[g - p.begin] = src;
      if (src != (int)g) atomicAdd(&p.state->block_changed, 1);
    } else if (src != (int)g) {
      const int slot = atomicAdd(&p.state->swap_count, 1);
      p.swap_extra[2 * slot + 0] = (int)g;
      p.swap_extra[2 * slot + 1] = src;
    }
  }
}

size_t panel_cluster_smem_bytes(int w, int rows_per_cta) {
  const size_t rp = (size_t)(rows_per_cta | 1);
  return (((size_t)w * rp + 1) & ~(size_t)1) * sizeof(double) + 32 * sizeof(CandSlot) +
         (size_t)(2 * 17 + kSub) * (w + 1) * sizeof(double) +
         (size_t)((rows_per_cta + 3) & ~3) * sizeof(int);
}

int panel_cluster_threads() { return kThreads; }

}  // namespace dp
