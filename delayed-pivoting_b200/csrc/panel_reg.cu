// Panel factorisation on one thread-block cluster with the sub-panel in
// registers (panels of up to 512 rows per CTA).
//
// Same contract and semantics as panel_cluster_kernel
// (delayed_lu/delayed_dgetrf.cpp:164-240: column partial-pivot search with
// first-index ties and NaN never winning, acceptance |alpha| > threshold,
// row swap, scaling by the reciprocal pivot, rank-1 update, stop at the first
// column without an acceptable pivot), with less work per column:
//   * every thread holds its rows' 8-column sub-panel slice in registers
//     (RPT rows per thread), so the swap, scaling and rank-1 update of a step
//     touch no shared memory;
//   * a step pushes one ~100-byte slot per CTA to every CTA of the cluster
//     (its candidate: magnitude, row, runner-up, reciprocal, source row and
//     the row's 8 sub-panel values; the owner of row k also pushes row k's
//     slice), then one hardware cluster barrier; every CTA then picks the
//     same winner and updates its own registers;
//   * the rest of each row (the finished L columns left of the sub-panel and
//     the columns right of it) does not change during a sub-panel, so rows
//     are moved there only at the sub-panel's end: every CTA replays the
//     sub-panel's swaps into a composite source map and pulls the content of
//     its moved rows - and the pivot rows for U12 = L11^{-1} A12 - from the
//     owning CTAs' shared memory (phase A), a second cluster barrier, then
//     writes them in place (phase B) and applies the rank-8 update of the
//     columns right of the sub-panel.
// Push buffers are indexed by step parity: a slot written at step s + 2 is
// written after the barrier of step s + 1, which every reader of step s
// passes only after finishing step s.  No spin-waits: the only waits are the
// hardware barriers.
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

constexpr int kT = 256;      // threads
constexpr int kW = kT / 32;  // warps
constexpr int kS = 8;        // sub-panel width
constexpr int kMaxC = 16;    // largest cluster

// One CTA's candidate (or row k) as pushed to every CTA.
struct __align__(16) Slot {
  double val;    // magnitude (>= 0)
  double sec;    // runner-up magnitude among the CTA's rows
  double inv;    // reciprocal of the candidate's entry in the current column
  int row;       // global row, -1 when the CTA has no candidate
  int orig;      // source row of its content (for the swap lists)
  double v[kS];  // the row over the sub-panel's columns
};

constexpr int kSlotChunks = (int)(sizeof(Slot) / sizeof(uint4));
static_assert(sizeof(Slot) % sizeof(uint4) == 0, "slots travel in 16-byte stores");

// offer() that also keeps the signed entry of the best row, whose reciprocal
// is then taken before the warp reduction instead of after it.
__device__ __forceinline__ void offer_x(LocalBest& b, double& bx, double x, int r) {
  const double v = fabs(x);
  if (v > b.val) {
    b.sec = b.val;
    b.val = v;
    b.row = r;
    bx = x;
  } else if (v > b.sec) {
    b.sec = v;
  }
}

struct Layout {
  double* sm;     // [w][RP] the panel slice
  Slot* slots;    // [2][kMaxC] candidates, by step parity and CTA rank
  Slot* kslot;    // [2] row k, by step parity
  Slot* stage;    // [kW] per-warp candidates, then [1] row k
  double* psave;  // [kS][W1] the sub-panel's pivot rows
  double* tmp;    // [2 kS][W1] pulled content of moved rows (by map entry)
  int* orig;      // [R] source row of each local row
  int* plist;     // [kS][2] (k, pivot row) of the sub-panel's steps
  int* own;       // [1 + 3 * 2 kS]: count, then (local row, source owner, source
                  // local row) of the moved rows this CTA owns
  int* ksrc;      // [2 kS]: (owner, local row) of the content of each step's row k
  unsigned long long* xbar;  // [2] exchange barriers, by step parity
};

__host__ __device__ inline size_t reg_align16(size_t bytes) { return (bytes + 15) & ~(size_t)15; }

__host__ __device__ inline size_t reg_layout(unsigned char* base, int w, int R, Layout* L) {
  const size_t rp = (size_t)(R | 1), w1 = (size_t)w + 1;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base ? base + off : nullptr;
    off += reg_align16(bytes);
    return p;
  };
  unsigned char* sm = take(sizeof(double) * (size_t)w * rp);
  unsigned char* slots = take(sizeof(Slot) * 2 * kMaxC);
  unsigned char* kslot = take(sizeof(Slot) * 2);
  unsigned char* stage = take(sizeof(Slot) * (kW + 1));
  unsigned char* psave = take(sizeof(double) * kS * w1);
  unsigned char* tmp = take(sizeof(double) * 2 * kS * w1);  // row q: map entry q
  unsigned char* orig = take(sizeof(int) * (size_t)R);
  unsigned char* plist = take(sizeof(int) * 2 * kS);
  unsigned char* own = take(sizeof(int) * (1 + 6 * kS));
  unsigned char* ksrc = take(sizeof(int) * 2 * kS);
  unsigned char* xbar = take(sizeof(unsigned long long) * 2);
  if (L) {
    L->sm = reinterpret_cast<double*>(sm);
    L->slots = reinterpret_cast<Slot*>(slots);
    L->kslot = reinterpret_cast<Slot*>(kslot);
    L->stage = reinterpret_cast<Slot*>(stage);
    L->psave = reinterpret_cast<double*>(psave);
    L->tmp = reinterpret_cast<double*>(tmp);
    L->orig = reinterpret_cast<int*>(orig);
    L->plist = reinterpret_cast<int*>(plist);
    L->own = reinterpret_cast<int*>(own);
    L->ksrc = reinterpret_cast<int*>(ksrc);
    L->xbar = reinterpret_cast<unsigned long long*>(xbar);
  }
  return off;
}

}  // namespace

template <int RPT>
__global__ void __launch_bounds__(kT, 1) panel_reg_kernel(PanelParams p) {
  // Every CTA reads the same word before any barrier or state write (a stop
  // is recorded only by an earlier kernel), so all of them leave together.
  if (p.gated && p.state->stop_k >= 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int w = p.end - p.begin;
  const int W1 = w + 1;
  const int R = p.rows_per_cta;
  const int RP = R | 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long row0 = (long long)p.begin + (long long)rank * R;
  const int rows_here = (int)max(0LL, min((long long)R, (long long)p.m - row0));
  Layout S;
  reg_layout(smem_raw, w, R, &S);
  double* const sm = S.sm;
  int* const orig = S.orig;

  // the slice arrives by asynchronous copies, all in flight at once
  for (int c = 0; c < w; ++c) {
    const double* src = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += kT) panel::cp_async8(sm + c * RP + r, src + r);
  }
  for (int r = tid; r < rows_here; r += kT) orig[r] = (int)(row0 + r);
  panel::cp_async_wait_all();
  if (rank == 0 && tid == 0) {
    p.state->stop_k = -1;
    p.state->swap_count = 0;
    p.state->block_changed = 0;
  }
  const unsigned xbar0 = panel::smem_addr(S.xbar);
  if (tid == 0) {
    panel::xbar_init(xbar0);
    panel::xbar_init(xbar0 + 8);
    panel::xbar_init_fence();
  }
  // every CTA's slice loaded and exchange barriers initialised before any
  // peer reads the one or writes to the other
  cluster.sync();

  // candidate of column 0
  LocalBest mine{0.0, -1, 0, 0.0};
  double mine_x = 0.0;  // signed entry of the candidate
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const int r = tid + i * kT;
    if (r < rows_here) offer_x(mine, mine_x, sm[r], r);
  }

  DecisionTally tally;  // rank 0, thread 0 records the decisions
  bool stopped = false, timed_out = false;
  bool pending = false;  // a cluster_arrive() awaits its cluster_wait()
  for (int base = 0; base < w && !stopped; base += kS) {
    const int send = min(base + kS, w);
    double x[RPT][kS];  // this thread's rows over the sub-panel's columns
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const int r = tid + i * kT;
#pragma unroll
      for (int t = 0; t < kS; ++t)
        x[i][t] = (r < rows_here && base + t < w) ? sm[(base + t) * RP + r] : 0.0;
    }
    int kd = send - base;  // steps executed in this sub-panel

#pragma unroll
    for (int j = 0; j < kS; ++j) {
      if (base + j >= w) break;
      const int s = base + j;
      const long long k = (long long)p.begin + s;
      const int par = s & 1;
      const bool positioned = (s == 0) && p.positioned;
      const int kl = (int)(k - row0);
      const bool own_k = kl >= 0 && kl < rows_here;

      const unsigned xb = xbar0 + 8u * (unsigned)par;
      if (tid == 0) panel::xbar_expect(xb, (unsigned)((C + 1) * sizeof(Slot)));

      // 1. this CTA's candidate: per-warp winners staged with their slices
      if (positioned) {
        mine = LocalBest{0.0, -1, 0, 0.0};
        if (own_k && tid == kl % kT) {
          mine = LocalBest{__longlong_as_double(0x7ff0000000000000ll), kl, 0, 0.0};
          mine_x = sm[kl];  // step 0: column 0 in shared memory is still current
        }
      }
      const double mine_inv = mine.row >= 0 ? 1.0 / mine_x : 0.0;
      const LocalBest wb = warp_lb(mine);
      if (wb.row >= 0 && tid == wb.row % kT) {
        Slot& st = S.stage[warp];
        const int wi = wb.row / kT;
#pragma unroll
        for (int i = 0; i < RPT; ++i)
          if (i == wi) {
#pragma unroll
            for (int t = 0; t < kS; ++t) st.v[t] = x[i][t];
          }
        st.inv = mine_inv;
        st.val = wb.val;
        st.sec = wb.sec;
        st.row = (int)(row0 + wb.row);
        st.orig = orig[wb.row];
      } else if (wb.row < 0 && lane == 0) {
        Slot& st = S.stage[warp];
        st.val = 0.0;
        st.sec = wb.sec;
        st.inv = 0.0;
        st.row = -1;
        st.orig = -1;
      }
      if (own_k && tid == kl % kT) {
        Slot& st = S.stage[kW];
        const int ki = kl / kT;
#pragma unroll
        for (int i = 0; i < RPT; ++i)
          if (i == ki) {
#pragma unroll
            for (int t = 0; t < kS; ++t) st.v[t] = x[i][t];
          }
        st.orig = orig[kl];
        st.row = (int)k;
      }
      __syncthreads();
      // 2. the CTA's winner among the warps, pushed to every CTA
      {
        const Slot* cs = S.stage + (lane & (kW - 1));
        const bool have = lane < kW && cs->row >= 0;
        double bv;
        int brow;
        warp_best(have ? cs->val : 0.0, have ? cs->row : 0x7fffffff, bv, brow);
        const double bsec = warp_max_pos(
            lane < kW ? ((have && cs->row == brow) ? cs->sec : (have ? cs->val : cs->sec)) : 0.0);
        const int wsel = __ffs(__ballot_sync(0xffffffffu, have && cs->row == brow)) - 1;
        if (warp == 0 && lane < C) {
          uint4 c[kSlotChunks];
          const uint4* src = reinterpret_cast<const uint4*>(S.stage + (wsel >= 0 ? wsel : 0));
#pragma unroll
          for (int i = 0; i < kSlotChunks; ++i) c[i] = src[i];
          if (wsel < 0) {  // no candidate: magnitude 0, row -1, reciprocal 0
            c[0].x = c[0].y = 0u;
            c[1] = make_uint4(0u, 0u, 0xffffffffu, 0xffffffffu);
          }
          const unsigned long long sb = (unsigned long long)__double_as_longlong(bsec);
          c[0].z = (unsigned)sb;
          c[0].w = (unsigned)(sb >> 32);
          const unsigned dst = panel::peer_addr(panel::smem_addr(S.slots + par * kMaxC + rank), lane);
          const unsigned bar = panel::peer_addr(xb, lane);
#pragma unroll
          for (int i = 0; i < kSlotChunks; ++i) panel::st_async16(dst + 16u * i, c[i], bar);
        }
        if (warp == 1 && own_k && lane < C) {
          const uint4* src = reinterpret_cast<const uint4*>(S.stage + kW);
          const unsigned dst = panel::peer_addr(panel::smem_addr(S.kslot + par), lane);
          const unsigned bar = panel::peer_addr(xb, lane);
#pragma unroll
          for (int i = 0; i < kSlotChunks; ++i) panel::st_async16(dst + 16u * i, src[i], bar);
        }
      }
      // every CTA's slot and row k's slice have arrived (use s >> 1 of this
      // parity's barrier)
      if (__syncthreads_or(!panel::xbar_wait(xb, (unsigned)(s >> 1) & 1u))) {
        if (tid == 0) p.state->status = kDeviceTimeout;
        timed_out = stopped = true;
        kd = 0;
        break;
      }

      // 3. same decision everywhere
      int wslot = -1;
      double wval = 0.0, wsec = 0.0;
      {
        const Slot* cs = S.slots + par * kMaxC + (lane < C ? lane : 0);
        const bool have = lane < C && cs->row >= 0;
        double bv;
        int brow;
        warp_best(have ? cs->val : 0.0, have ? cs->row : 0x7fffffff, bv, brow);
        wsec = warp_max_pos(lane < C ? ((have && cs->row == brow) ? cs->sec
                                                                 : (have ? cs->val : cs->sec))
                                     : 0.0);
        if (brow != 0x7fffffff) {
          wslot = __ffs(__ballot_sync(0xffffffffu, have && cs->row == brow)) - 1;
          wval = bv;
        }
      }
      if (rank == 0 && tid == 0 && !positioned) tally.note(k, wval, wsec);
      const bool stop = !positioned && !(wslot >= 0 && wval > p.threshold);
      if (stop) {
        if (rank == 0 && tid == 0) p.state->stop_k = (int)k;
        kd = j;
        stopped = true;
        break;
      }
      const Slot& ws = S.slots[par * kMaxC + wslot];
      const long long prow = ws.row;
      if (rank == 0 && tid == 0 && !positioned) p.ipiv[k] = (int)prow;
      if (tid == 0) {
        S.plist[2 * j] = (int)k;
        S.plist[2 * j + 1] = (int)prow;
      }
      if (tid < kS && base + tid < w) S.psave[j * W1 + base + tid] = ws.v[tid];
      double pv[kS];
#pragma unroll
      for (int t = 0; t < kS; ++t) pv[t] = ws.v[t];
      const double inv = ws.inv;

      // 4. swap: row k takes the pivot row, the pivot row's place row k
      const int pl = (int)(prow - row0);
      const bool swap_p = pl >= 0 && pl < rows_here && prow != k;
      if (own_k && tid == kl % kT) {
        const int ki = kl / kT;
#pragma unroll
        for (int i = 0; i < RPT; ++i)
          if (i == ki) {
#pragma unroll
            for (int t = 0; t < kS; ++t) x[i][t] = pv[t];
          }
        orig[kl] = ws.orig;
      }
      if (swap_p && tid == pl % kT) {
        const Slot& kr = S.kslot[par];
        const int pi = pl / kT;
#pragma unroll
        for (int i = 0; i < RPT; ++i)
          if (i == pi) {
#pragma unroll
            for (int t = 0; t < kS; ++t) x[i][t] = kr.v[t];
          }
        orig[pl] = kr.orig;
      }

      // 5. scale and update the rows below k; next column's candidate
      mine = LocalBest{0.0, -1, 0, 0.0};
#pragma unroll
      for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * kT;
        if (r >= rows_here || row0 + r <= k) continue;
        const double l = x[i][j] * inv;
        x[i][j] = l;
#pragma unroll
        for (int t = j + 1; t < kS; ++t) x[i][t] = fma(-l, pv[t], x[i][t]);
        if (j + 1 < kS && s + 1 < send) offer_x(mine, mine_x, x[i][j + 1 < kS ? j + 1 : 0], r);
      }
    }

    // ---- end of the sub-panel: kd steps executed at [base, base + kd) ----
    if (kd == 0) break;  // stopped at its first step: nothing moved
    // a. the register slices back to shared memory
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const int r = tid + i * kT;
      if (r < rows_here) {
#pragma unroll
        for (int t = 0; t < kS; ++t)
          if (base + t < w) sm[(base + t) * RP + r] = x[i][t];
      }
    }
    // b. composite source map of the sub-panel's swaps (the same everywhere):
    //    lane q of warp 0 takes position k_q (q < kd) or p_{q - kd} and traces
    //    it back through the swaps to the row whose content it holds now.
    //    Kept: where the content of each k_q is (the sub-panel's pivot rows,
    //    for U12) and, compacted by a ballot, the moved positions this CTA
    //    owns (a pivot row that is also a later step's row k once), each with
    //    its source's owner and local row
    if (warp == 0) {
      const bool on = lane < 2 * kd;
      int x = on ? S.plist[lane < kd ? 2 * lane : 2 * (lane - kd) + 1] : 0;
      const int pos = x;
      for (int t = kd - 1; t >= 0 && on; --t) {
        const int a = S.plist[2 * t], b = S.plist[2 * t + 1];
        x = x == a ? b : (x == b ? a : x);
      }
      const int so = on ? (int)((x - p.begin) / R) : 0;
      const int sl = on ? (int)(x - p.begin - (long long)so * R) : 0;
      if (lane < kd) {
        S.ksrc[2 * lane] = so;
        S.ksrc[2 * lane + 1] = sl;
      }
      bool keep = on && x != pos && pos >= row0 && pos < row0 + rows_here;
      for (int q = 0; q < 2 * kS; ++q) {  // first occurrence of each position
        const int other = __shfl_sync(0xffffffffu, pos, q);
        if (q < lane && q < 2 * kd && other == pos) keep = false;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int at = __popc(bal & ((1u << lane) - 1u));
        S.own[1 + 3 * at] = (int)(pos - row0);
        S.own[2 + 3 * at] = so;
        S.own[3 + 3 * at] = sl;
      }
      if (lane == 0) S.own[0] = __popc(bal);
    }
    __syncthreads();
    const int nown = S.own[0];
    // the owners' writes of the previous sub-panel end are visible
    if (pending) {
      panel::cluster_wait();
      pending = false;
    }
    const int ncol_out = base + (w - send);  // columns outside the sub-panel
    auto out_col = [&](int c) { return c < base ? c : send + (c - base); };
    // c. phase A: the moved rows of this CTA (into tmp, row q for own entry
    //    q) and the pivot rows' columns right of the sub-panel (into psave),
    //    read from their owners' shared memory; every (row, column) element
    //    is an independent load, four per thread in flight
    {
      const int na = nown * ncol_out;
      for (int e0 = tid; e0 < na; e0 += 4 * kT) {
        double v[4];
        int at[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int e = e0 + u * kT;
          at[u] = -1;
          if (e < na) {
            const int q = e / ncol_out, c = e - q * ncol_out;
            const double* src = cluster.map_shared_rank(sm, S.own[2 + 3 * q]);
            v[u] = src[out_col(c) * RP + S.own[3 + 3 * q]];
            at[u] = q * W1 + c;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (at[u] >= 0) S.tmp[at[u]] = v[u];
      }
    }
    if (send < w) {
      const int nr = w - send, np = kd * nr;
      for (int e0 = tid; e0 < np; e0 += 4 * kT) {
        double v[4];
        int at[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int e = e0 + u * kT;
          at[u] = -1;
          if (e < np) {
            const int t = e / nr, c = send + (e - t * nr);
            const double* src = cluster.map_shared_rank(sm, S.ksrc[2 * t]);
            v[u] = src[c * RP + S.ksrc[2 * t + 1]];
            at[u] = t * W1 + c;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (at[u] >= 0) S.psave[at[u]] = v[u];
      }
    }
    cluster.sync();  // every CTA has read what it needs before anyone overwrites
    // d. phase B: moved rows take their sources' content
    for (int e = tid; e < nown * ncol_out; e += kT) {
      const int q = e / ncol_out, c = e - q * ncol_out;
      sm[out_col(c) * RP + S.own[1 + 3 * q]] = S.tmp[q * W1 + c];
    }
    if (send >= w) break;  // no columns right of the sub-panel
    __syncthreads();       // psave and the moved rows complete
    // e. U12 = L11^{-1} A12 of the sub-panel, one column per thread
    for (int c = send + tid; c < w; c += kT) {
      double u[kS];
#pragma unroll
      for (int q = 0; q < kS; ++q) u[q] = q < kd ? S.psave[q * W1 + c] : 0.0;
#pragma unroll
      for (int q = 1; q < kS; ++q) {
        if (q < kd) {
#pragma unroll
          for (int t = 0; t < q; ++t) u[q] = fma(-S.psave[q * W1 + base + t], u[t], u[q]);
          S.psave[q * W1 + c] = u[q];
        }
      }
    }
    __syncthreads();
    const long long first = (long long)p.begin + base;  // global row of the first pivot
    const int ncol = w - send;
    // the solved rows to the pivot rows of this CTA
    for (int e = tid; e < kd * ncol; e += kT) {
      const int q = e / ncol, c = send + (e - q * ncol);
      const long long g = first + q;
      if (g >= row0 && g < row0 + rows_here) sm[c * RP + (int)(g - row0)] = S.psave[q * W1 + c];
    }
    // f. rank-kd update of the rows below the sub-panel's pivots on the FP64
    //    tensor path (mma.sync.m16n8k4, the kd <= 8 steps as two k4 steps):
    //    warp w takes rows [32 w + 256 i, + 32) in 16 x 8 tiles over the
    //    columns [send, w), C read from and written to shared memory; rows
    //    above the sub-panel's last pivot or beyond the CTA's keep their
    //    values.  Then the next sub-panel's first candidate.
    {
      const double* __restrict__ ps = S.psave;
      const int g = lane >> 2, t4 = lane & 3;
      const int lim = (int)max(0LL, min((long long)rows_here, first + kd - row0));
      const int ncol = w - send;
#pragma unroll
      for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const int rb = warp * 32 + i * kT + mt * 16;
          if (rb >= rows_here || rb + 16 <= lim) continue;  // (warp-uniform)
          const bool ok0 = rb + g < rows_here, ok1 = rb + g + 8 < rows_here;
          double a[2][2];
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            const int k = 4 * ks + t4;
            a[ks][0] = (k < kd && ok0) ? -sm[(base + k) * RP + rb + g] : 0.0;
            a[ks][1] = (k < kd && ok1) ? -sm[(base + k) * RP + rb + g + 8] : 0.0;
          }
          const bool st0 = ok0 && rb + g >= lim, st1 = ok1 && rb + g + 8 >= lim;
          for (int c0 = 0; c0 < ncol; c0 += 8) {
            double b[2];
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              const int k = 4 * ks + t4;
              b[ks] = (k < kd && c0 + g < ncol) ? ps[k * W1 + send + c0 + g] : 0.0;
            }
            const int ca = send + c0 + 2 * t4;  // this lane's columns ca, ca + 1
            double c[4];
            c[0] = (ok0 && ca < w) ? sm[ca * RP + rb + g] : 0.0;
            c[1] = (ok0 && ca + 1 < w) ? sm[(ca + 1) * RP + rb + g] : 0.0;
            c[2] = (ok1 && ca < w) ? sm[ca * RP + rb + g + 8] : 0.0;
            c[3] = (ok1 && ca + 1 < w) ? sm[(ca + 1) * RP + rb + g + 8] : 0.0;
            panel::mma_f64(c, a[0][0], a[0][1], b[0]);
            panel::mma_f64(c, a[1][0], a[1][1], b[1]);
            if (st0 && ca < w) sm[ca * RP + rb + g] = c[0];
            if (st0 && ca + 1 < w) sm[(ca + 1) * RP + rb + g] = c[1];
            if (st1 && ca < w) sm[ca * RP + rb + g + 8] = c[2];
            if (st1 && ca + 1 < w) sm[(ca + 1) * RP + rb + g + 8] = c[3];
          }
        }
    }
    __syncthreads();  // every warp's tiles are stored
    mine = LocalBest{0.0, -1, 0, 0.0};
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const int r = tid + i * kT;
      if (r < rows_here && row0 + r >= first + kd) offer_x(mine, mine_x, sm[send * RP + r], r);
    }
    __syncthreads();  // the next sub-panel's columns are final in shared memory
    // released to the readers of the next sub-panel end (phase A); the
    // steps in between exchange through the transaction barriers alone
    panel::cluster_arrive();
    pending = true;
  }
  // No CTA may exit while a peer could still read its shared memory, and
  // rows were written by other threads than those writing them back.
  if (pending)
    panel::cluster_wait();
  else
    cluster.sync();
  if (timed_out) return;
  if (rank == 0 && tid == 0) tally.flush(p.state);

#pragma unroll 4
  for (int c = 0; c < w; ++c) {
    double* dst = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += kT) dst[r] = sm[c * RP + r];
  }
  // Swap lists: whole warps walk the rows together, so that the moved rows
  // below the block take their slots with one atomic per warp.
  int changed = 0;
  for (int r0w = warp * 32; r0w < rows_here; r0w += kT) {
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

size_t panel_reg_smem_bytes(int w, int rows_per_cta) {
  return reg_layout(nullptr, w, rows_per_cta, nullptr);
}

// Up to 512 rows per CTA: at 1024 (four rows per thread) the shared-memory
// cluster panel was measured faster per column (3.9 against 4.3 us).
int panel_reg_max_rows() { return 2 * kT; }

const void* panel_reg_kernel_for(int rows_per_cta) {
  if (rows_per_cta <= kT) return (const void*)panel_reg_kernel<1>;
  if (rows_per_cta <= 2 * kT) return (const void*)panel_reg_kernel<2>;
  return nullptr;
}

}  // namespace dp
