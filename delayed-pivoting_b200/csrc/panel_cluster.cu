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
#include "panel_argmax.cuh"

namespace cg = cooperative_groups;

namespace dp {

namespace {

using panel::LocalBest;
using panel::offer;
using panel::warp_best;
using panel::warp_lb;
using panel::warp_max_pos;
using panel::cp_async8;
using panel::cp_async_wait_all;

constexpr int kThreads = 256;
constexpr int kSub = 8;  // sub-panel width
constexpr int kMaxW = 128;  // widest panel (the TRSM's limit)
constexpr int kPushPer = (kMaxW + 1 + 31) / 32;  // pushed row elements per lane

struct __align__(16) CandSlot {
  double val;
  int row;     // global row, -1 when the CTA has no candidate
  int pad;
  double inv;  // reciprocal of the candidate's entry in the current column
  double sec;  // runner-up magnitude among the CTA's rows (near-tie detector)
};

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

  // the slice arrives by asynchronous copies, all in flight at once
  for (int c = 0; c < w; ++c) {
    const double* src = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += blockDim.x) cp_async8(sm + c * RP + r, src + r);
  }
  for (int r = tid; r < rows_here; r += blockDim.x) orig[r] = (int)(row0 + r);
  cp_async_wait_all();
  if (rank == 0 && tid == 0) {
    p.state->stop_k = -1;
    p.state->swap_count = 0;
    p.state->block_changed = 0;
  }
  __syncthreads();

  LocalBest mine{0.0, -1, 0, 0.0};
  {
    const int kl0 = (int)((long long)p.begin - row0);
    for (int r = max(0, kl0) + tid; r < rows_here; r += blockDim.x) offer(mine, fabs(sm[r]), r);
  }

  // End of a sub-panel that executed kd steps at [base, base + kd): solve its
  // pivot rows for the columns [send, w), give them to the pivot rows held
  // here and update the rows below; each updating thread also finds its
  // candidate of column send (the next step's search, rows below the last
  // pivot only).  Called with kd = 0 only when the panel stops.
  auto sub_panel_end = [&](int kd, int base, int send) {
    __syncthreads();  // psave complete, this CTA's rows updated
    mine = LocalBest{0.0, -1, 0, 0.0};
    if (kd == 0) return;
    // U12 = L11^{-1} A12 of the sub-panel, one column per thread, in registers
    for (int c = send + tid; c < w; c += blockDim.x) {
      double u[kSub];
#pragma unroll
      for (int j = 0; j < kSub; ++j) u[j] = j < kd ? psave[j * W1 + c] : 0.0;
#pragma unroll
      for (int j = 1; j < kSub; ++j) {
        if (j < kd) {
#pragma unroll
          for (int t = 0; t < j; ++t) u[j] = fma(-psave[j * W1 + base + t], u[t], u[j]);
          psave[j * W1 + c] = u[j];
        }
      }
    }
    __syncthreads();
    const long long first = (long long)p.begin + base;  // global row of the first pivot
    const int ncol = w - send;
    // the solved rows to the pivot rows of this CTA, spread over the threads
    for (int e = tid; e < kd * ncol; e += blockDim.x) {
      const int j = e / ncol, c = send + (e - j * ncol);
      const long long g = first + j;
      if (g >= row0 && g < row0 + rows_here) sm[c * RP + (int)(g - row0)] = psave[j * W1 + c];
    }
    const double* __restrict__ ps = psave;
    for (int r = tid; r < rows_here; r += blockDim.x) {
      const long long g = row0 + r;
      if (g < first + kd) continue;
      double* __restrict__ row = sm + r;
      double l[kSub];
#pragma unroll
      for (int t = 0; t < kSub; ++t) l[t] = t < kd ? row[(base + t) * RP] : 0.0;
      {
        // column send first: the next step's candidate
        double x = row[send * RP];
#pragma unroll
        for (int t = 0; t < kSub; ++t)
          if (t < kd) x = fma(-l[t], ps[t * W1 + send], x);
        row[send * RP] = x;
        offer(mine, fabs(x), r);
      }
#pragma unroll 4
      for (int c = send + 1; c < w; ++c) {
        double x = row[c * RP];
#pragma unroll
        for (int t = 0; t < kSub; ++t)
          if (t < kd) x = fma(-l[t], ps[t * W1 + c], x);
        row[c * RP] = x;
      }
    }
  };

  DecisionTally tally;  // rank 0, thread 0 records the decisions
  for (int s = 0; s < w; ++s) {
    const long long k = (long long)p.begin + s;
    const int par = s & 1;
    const bool positioned = (s == 0) && p.positioned;
    const int kl = (int)(k - row0);
    const bool own_k = kl >= 0 && kl < rows_here;

    // 1. CTA candidate (every thread reduces the per-warp results itself).
    if (positioned) {
      mine = LocalBest{0.0, -1, 0, 0.0};
      if (own_k && tid == 0)
        mine = LocalBest{__longlong_as_double(0x7ff0000000000000ll), kl, 0, 0.0};
    }
    mine = warp_lb(mine);
    if (lane == 0) red[warp] = mine;
    __syncthreads();
    const LocalBest cb = warp_lb(lane < nwarps ? red[lane] : LocalBest{0.0, -1, 0, 0.0});

    // 2. Push (value, row), the candidate row and row k into every CTA.
    {
      double* my_stc = stc + (par * 16 + rank) * W1;
      double* my_stk = stk + par * W1;
      // warp w pushes to CTAs w, w + nwarps, ...; its lanes walk the row
      // each lane reads its elements of both rows once, then stores them
      // to every destination of its warp
      if (warp < C && (cb.row >= 0 || own_k)) {
        double cv[kPushPer], kv[kPushPer];
#pragma unroll
        for (int u = 0; u < kPushPer; ++u) {
          const int j = lane + 32 * u;
          cv[u] = (cb.row >= 0 && j < W1) ? (j < w ? sm[j * RP + cb.row] : (double)orig[cb.row])
                                          : 0.0;
          kv[u] = (own_k && j < W1) ? (j < w ? sm[j * RP + kl] : (double)orig[kl]) : 0.0;
        }
        for (int dest = warp; dest < C; dest += nwarps) {
          double* rc = cluster.map_shared_rank(my_stc, dest);
          double* rk = cluster.map_shared_rank(my_stk, dest);
#pragma unroll
          for (int u = 0; u < kPushPer; ++u) {
            const int j = lane + 32 * u;
            if (j < W1) {
              if (cb.row >= 0) rc[j] = cv[u];
              if (own_k) rk[j] = kv[u];
            }
          }
        }
      }
      if (tid < C) {
        CandSlot cs;
        cs.val = cb.row >= 0 ? cb.val : 0.0;
        cs.row = cb.row >= 0 ? (int)(row0 + cb.row) : -1;
        cs.pad = 0;
        cs.inv = cb.row >= 0 ? 1.0 / sm[s * RP + cb.row] : 0.0;
        cs.sec = cb.sec;
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
      // runner-up over the cluster: the winner slot's runner-up, every other slot's best
      win.sec = warp_max_pos((c.row >= 0 && c.row == brow) ? c.sec
                                                           : (c.row >= 0 ? c.val : c.sec));
      if (brow != 0x7fffffff) {
        // the slot holding the winner (global rows are unique)
        const int src = __ffs(__ballot_sync(0xffffffffu, c.row == brow && lane < C)) - 1;
        win.val = bv;
        win.row = brow;
        win.inv = __shfl_sync(0xffffffffu, c.inv, max(src, 0));
      }
    }
    if (rank == 0 && tid == 0 && !positioned) tally.note(k, win.val, win.sec);
    const bool stop = !positioned && !(win.row >= 0 && win.val > p.threshold);
    if (stop) {
      if (rank == 0 && tid == 0) p.state->stop_k = (int)k;
      // the columns right of the sub-panel take its executed steps
      const int base = (s / kSub) * kSub, send = min(base + kSub, w);
      if (send < w) sub_panel_end(s - base, base, send);
      break;
    }
    const long long prow_g = win.row;
    const int owner_p = (int)(prow_g - p.begin) / R;
    const double* __restrict__ pr = stc + (par * 16 + owner_p) * W1;
    const double* __restrict__ kr = stk + par * W1;
    const int pl = (int)(prow_g - row0);
    const bool swap_p = pl >= 0 && pl < rows_here && prow_g != k;
    if (rank == 0 && tid == 0 && !positioned) p.ipiv[k] = (int)prow_g;
    const int base = (s / kSub) * kSub, send = min(base + kSub, w);
    for (int j = tid; j < W1; j += blockDim.x) psave[(s - base) * W1 + j] = pr[j];

    // 4. Row k takes the pivot row and row pl row k's old content (columns
    //    outside [s, send): the updating thread writes those), spread over
    //    the threads; then every thread swaps, scales and updates its own
    //    rows, reading row pl's old values from the pushed row k.  The next
    //    column's candidate is on the way.
    if (own_k)
      for (int j = tid; j < W1; j += blockDim.x) {
        if (j < w) sm[j * RP + kl] = pr[j];
        else orig[kl] = (int)pr[w];
      }
    if (swap_p)
      for (int j = tid; j < W1; j += blockDim.x) {
        if (j < w) {
          if (j < s || j >= send) sm[j * RP + pl] = kr[j];
        } else {
          orig[pl] = (int)kr[w];
        }
      }
    const double inv = win.inv;
    double pv[kSub];  // pivot row over the sub-panel's columns [s, send)
    pv[0] = 0.0;
#pragma unroll
    for (int t = 1; t < kSub; ++t) pv[t] = s + t < send ? pr[s + t] : 0.0;
    mine = LocalBest{0.0, -1, 0, 0.0};
#pragma unroll 2
    for (int r = max(0, kl + 1) + tid; r < rows_here; r += blockDim.x) {
      double* __restrict__ row = sm + r;
      const bool from_k = swap_p && r == pl;
      // row pl's old values are the pushed row k: one load per element either way
      const double* __restrict__ xs = from_k ? kr + s : row + s * RP;
      const int xstride = from_k ? 1 : RP;
      double x[kSub];
#pragma unroll
      for (int t = 0; t < kSub; ++t) x[t] = s + t < send ? xs[t * xstride] : 0.0;
      const double l = x[0] * inv;
      row[s * RP] = l;
#pragma unroll
      for (int t = 1; t < kSub; ++t)
        if (s + t < send) {  // columns past the sub-panel wait for its rank-kSub update
          x[t] = fma(-l, pv[t], x[t]);
          row[(s + t) * RP] = x[t];
        }
      if (s + 1 < send) offer(mine, fabs(x[1]), r);
    }
    if (s + 1 == send && send < w) sub_panel_end(s + 1 - base, base, send);
  }
  // Rows were swapped and updated by other threads than those writing them
  // back, and no CTA may exit while a peer could still push into it.
  cluster.sync();
  if (rank == 0 && tid == 0) tally.flush(p.state);

#pragma unroll 4
  for (int c = 0; c < w; ++c) {
    double* dst = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += blockDim.x) dst[r] = sm[c * RP + r];
  }
  // Swap lists: whole warps walk the rows together, so that the moved rows
  // below the block take their slots with one atomic per warp.
  int changed = 0;
  for (int r0w = warp * 32; r0w < rows_here; r0w += blockDim.x) {
    const int r = r0w + lane;
    const long long g = row0 + r;
    const int src = r < rows_here ? orig[r] : (int)g;
    if (r < rows_here && g < p.end) {
      p.swap_block[g - p.begin] = src;
      changed += src != (int)g;
    }
    const bool moved = r < rows_here && g >= p.end && src != (int)g;
    const unsigned bal = __ballot_sync(0xffffffffu, moved);
    if (bal) {
      int slot = 0;
      if (lane == 0) slot = atomicAdd(&p.state->swap_count, __popc(bal));
      slot = __shfl_sync(0xffffffffu, slot, 0) + __popc(bal & ((1u << lane) - 1u));
      if (moved) {
        p.swap_extra[2 * slot + 0] = (int)g;
        p.swap_extra[2 * slot + 1] = src;
      }
    }
  }
  changed = __reduce_add_sync(0xffffffffu, changed);
  if (lane == 0 && changed) atomicAdd(&p.state->block_changed, changed);
}

size_t panel_cluster_smem_bytes(int w, int rows_per_cta) {
  const size_t rp = (size_t)(rows_per_cta | 1);
  return (((size_t)w * rp + 1) & ~(size_t)1) * sizeof(double) + 32 * sizeof(CandSlot) +
         (size_t)(2 * 17 + kSub) * (w + 1) * sizeof(double) +
         (size_t)((rows_per_cta + 3) & ~3) * sizeof(int);
}

int panel_cluster_threads() { return kThreads; }

}  // namespace dp
