// Panel factorisation of the delayed-pivoting LU on many SMs at once.
//
// Follows the inner loop of delayed_lu/delayed_dgetrf.cpp:164-240 (and its
// GPU twin delayed_lu_cuda/delayed_dgetrf_cuda.cu:264-350) for the panel
// columns [begin, end):
//   column partial-pivot search (first index on ties, NaN never wins)
//   acceptance test |alpha| > threshold (threshold 0 == the reference's
//     `!(alpha > 0.0)`, delayed_dgetrf.cpp:178)
//   row swap inside the panel columns (the rest of each row is swapped later
//     by the laswp kernel from the swap list this kernel writes)
//   scale by the reciprocal of the pivot (delayed_dgetrf.cpp:225-227)
//   rank-1 update of the remaining panel columns (delayed_dgetrf.cpp:233-239)
// When a column has no acceptable pivot the kernel stops at that step k,
// records state->stop_k = k and leaves the fallback to the host driver.
//
// B200 layout: rows [begin, m) are split into G contiguous chunks of R rows,
// one per CTA; each CTA keeps its R x w slice of the panel in shared memory
// for the whole launch, so the panel crosses HBM once in and once out.  The
// only cross-CTA traffic per column is one 16-byte candidate and one row of w
// doubles, exchanged through L2 with tagged words (no atomics on the hot
// path): every CTA publishes its local argmax, every CTA reads all G
// candidates and reaches the same decision.  Launched cooperatively so all G
// CTAs are co-resident; every wait is bounded (kSpinLimitNs).
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int kPanelThreads = 256;
constexpr int kSlots = 4;  // exchange slots, indexed by step mod 4
constexpr int kMaxSlotsPerLane = 5;  // ceil(max CTAs (<= 160) / 32)
// Mailboxes: mbox[parity][q][reader][writer] holds the writer's tagged
// candidate (2 words, 16 bytes).  Every CTA pushes its candidate into every
// reader's mailbox and polls only its own, contiguous mailbox, so each line
// has exactly one reader and no CTA spins on a line another CTA is writing
// for everyone (which delayed the writers' stores by microseconds).
constexpr int kMboxWords = 2;

struct __align__(16) Best {
  double val;
  int row;  // local row, -1 when none
  int pad;
};

__device__ __forceinline__ Best best_of(Best a, Best b) {
  // larger value wins; ties (and equal values) go to the smaller row; a
  // candidate with row -1 never wins against a real one of equal value.
  if (b.row < 0) return a;
  if (a.row < 0) return b;
  if (b.val > a.val) return b;
  if (b.val == a.val && b.row < a.row) return b;
  return a;
}

__device__ __forceinline__ Best warp_best(Best v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    Best o;
    o.val = __shfl_down_sync(0xffffffffu, v.val, off);
    o.row = __shfl_down_sync(0xffffffffu, v.row, off);
    o.pad = 0;
    v = best_of(v, o);
  }
  return v;
}

// row[j * stride] = src[j] for j < w, loads of a batch before its stores.
__device__ __forceinline__ void copy_row(double* __restrict__ row, const double* __restrict__ src,
                                         int w, int stride) {
  int j = 0;
  for (; j + 8 <= w; j += 8) {
    double x[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) x[b] = src[j + b];
#pragma unroll
    for (int b = 0; b < 8; ++b) row[(size_t)(j + b) * stride] = x[b];
  }
  for (; j < w; ++j) row[(size_t)j * stride] = src[j];
}

}  // namespace

__global__ void __launch_bounds__(kPanelThreads, 1)
panel_factor_kernel(PanelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int w = p.end - p.begin;
  const int R = p.rows_per_cta;
  const int G = gridDim.x;
  const int cta = blockIdx.x;
  const int tid = threadIdx.x;
  const long long row0 = (long long)p.begin + (long long)cta * R;  // global row of local row 0
  const int rows_here = (int)min((long long)R, (long long)p.m - row0);
  const int RP = R | 1;  // odd column stride: a row read across columns hits distinct banks

  double* sm = reinterpret_cast<double*>(smem_raw);   // [w][RP]
  double* prow = sm + (size_t)w * RP;                 // [w + 1] pivot row (+orig)
  double* krow = prow + (w + 1);                      // [w + 1] old row k (+orig)
  int* orig = reinterpret_cast<int*>(krow + (w + 1));  // [R] source row of each local row
  __shared__ Best red[kPanelThreads / 32];
  __shared__ int s_flag[4];  // 0: winner row (global), 1: stop, 2: winner cta, 3: abort

  const size_t mbox_q = (size_t)p.max_ctas * p.max_ctas * kMboxWords;  // words per (parity, q)
  unsigned long long* mbox = p.slots + (size_t)(p.parity & 1) * kSlots * mbox_q;
  double* xdata = p.xdata;  // [kSlots][max_ctas][w_max + 1]
  double* rowk = p.rowk;    // [kSlots][w_max + 1]
  const int xs = p.w_max + 1;

  // Zero the mailboxes of readers cta, cta + G, ... in the other parity
  // buffer, which the next launch uses; no CTA of this launch touches it.
  {
    unsigned long long* other = p.slots + (size_t)((p.parity + 1) & 1) * kSlots * mbox_q;
    for (int rd = cta; rd < p.max_ctas; rd += G) {
      for (int q = 0; q < kSlots; ++q) {
        unsigned long long* box = other + q * mbox_q + (size_t)rd * p.max_ctas * kMboxWords;
        for (int i = tid; i < p.max_ctas * kMboxWords; i += blockDim.x) box[i] = 0ull;
      }
    }
  }
  if (cta == 0 && tid == 0) {
    p.state->stop_k = -1;
    p.state->swap_count = 0;
    p.state->block_changed = 0;
    __threadfence();
  }

  // Load the panel slice.
  for (int c = 0; c < w; ++c) {
    const double* src = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += blockDim.x) sm[(size_t)c * RP + r] = src[r];
  }
  for (int r = tid; r < rows_here; r += blockDim.x) orig[r] = (int)(row0 + r);
  __syncthreads();

  const int lane = tid & 31, warp = tid >> 5;
  bool aborted = false;

  // Local candidate of column 0 (later columns are found inside the rank-1
  // update of the previous step).  Strict '>' from an initial magnitude of
  // 0: zeros and NaN never become candidates; the first of equal magnitudes
  // stays (reference: idamax / delayed_dgetrf_cuda.cu:13-20).
  Best mine{0.0, -1, 0};
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

  for (int s = 0; s < w; ++s) {
    const long long k = (long long)p.begin + s;
    const int q = s & (kSlots - 1);
    const unsigned long long tb = (unsigned long long)(((s >> 2) & 1) ^ 1);
    const bool positioned = (s == 0) && p.positioned;
    const int kl = (int)(k - row0);  // local index of row k (valid if 0 <= kl < rows_here)
    const bool own_k = kl >= 0 && kl < rows_here;

    // 1. CTA candidate for column s.
    if (positioned) {
      mine = Best{0.0, -1, 0};
      if (own_k && tid == 0) mine = Best{__longlong_as_double(0x7ff0000000000000ll), kl, 0};
    }
    mine = warp_best(mine);
    if (lane == 0) red[warp] = mine;
    __syncthreads();

    // 2-4. Warp 0: publish, gather all G candidates (bounded wait), fetch the
    // pivot row.  One warp, one fence, no CTA barrier on the critical path.
    if (warp == 0) {
      Best cb = lane < (blockDim.x >> 5) ? red[lane] : Best{0.0, -1, 0};
      cb = warp_best(cb);
      cb.val = __shfl_sync(0xffffffffu, cb.val, 0);
      cb.row = __shfl_sync(0xffffffffu, cb.row, 0);
      double* xd = xdata + ((size_t)q * p.max_ctas + cta) * xs;
      if (cb.row >= 0) {
        for (int j = lane; j < w; j += 32) __stcg(xd + j, sm[(size_t)j * RP + cb.row]);
        if (lane == 0) __stcg(xd + w, (double)orig[cb.row]);
      }
      if (own_k) {
        double* rk = rowk + (size_t)q * xs;
        for (int j = lane; j < w; j += 32) __stcg(rk + j, sm[(size_t)j * RP + kl]);
        if (lane == 0) __stcg(rk + w, (double)orig[kl]);
      }
      fence_acq_rel_gpu();
      __syncwarp();
      {
        const unsigned long long vbits =
            cb.row >= 0 ? (unsigned long long)__double_as_longlong(cb.val) : 0ull;
        const unsigned long long grow =
            cb.row >= 0 ? (unsigned long long)(row0 + cb.row) : 0x7fffffffull;
        unsigned long long* boxes = mbox + q * mbox_q + (size_t)cta * kMboxWords;
        for (int rd = lane; rd < G; rd += 32)
          st_volatile_v2u64(boxes + (size_t)rd * p.max_ctas * kMboxWords, (vbits << 1) | tb,
                            (grow << 1) | tb);
      }

      // Each lane owns mailbox entries lane, lane + 32, ... (at most
      // kMaxSlotsPerLane) and re-reads all of its pending ones per round, so
      // a round costs one L2 round trip however many entries are late.
      unsigned long long best_bits = 0ull;
      long long best_row = 0x7fffffffll;
      bool have = false;
      const unsigned long long t0 = globaltimer_ns();
      bool timeout = false;
      unsigned pending = 0;
#pragma unroll
      for (int u = 0; u < kMaxSlotsPerLane; ++u)
        if (lane + 32 * u < G) pending |= 1u << u;
      unsigned int rounds = 0;
      while (pending) {
        unsigned long long kv[kMaxSlotsPerLane], kr[kMaxSlotsPerLane];
#pragma unroll
        for (int u = 0; u < kMaxSlotsPerLane; ++u) {
          if (pending & (1u << u)) {
            const unsigned long long* sl =
                mbox + q * mbox_q + ((size_t)cta * p.max_ctas + lane + 32 * u) * kMboxWords;
            ld_volatile_v2u64(sl, kv[u], kr[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < kMaxSlotsPerLane; ++u) {
          if ((pending & (1u << u)) && (kv[u] & 1ull) == tb && (kr[u] & 1ull) == tb) {
            pending &= ~(1u << u);
            const unsigned long long vb = kv[u] >> 1;
            const long long rr = (long long)(kr[u] >> 1);
            if (rr != 0x7fffffffll &&
                (!have || vb > best_bits || (vb == best_bits && rr < best_row))) {
              best_bits = vb;
              best_row = rr;
              have = true;
            }
          }
        }
        if (pending && ((++rounds) & 63u) == 0u) {
          if (globaltimer_ns() - t0 > kSpinLimitNs || ld_volatile_i32(&p.state->status) != kOk) {
            timeout = true;
            break;
          }
        }
      }
      const bool any_timeout = __any_sync(0xffffffffu, timeout);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long ob = __shfl_down_sync(0xffffffffu, best_bits, off);
        const long long orr = __shfl_down_sync(0xffffffffu, best_row, off);
        const int oh = __shfl_down_sync(0xffffffffu, (int)have, off);
        if (oh && (!have || ob > best_bits || (ob == best_bits && orr < best_row))) {
          best_bits = ob;
          best_row = orr;
          have = true;
        }
      }
      best_bits = __shfl_sync(0xffffffffu, best_bits, 0);
      best_row = __shfl_sync(0xffffffffu, best_row, 0);
      have = __shfl_sync(0xffffffffu, (int)have, 0) != 0;
      fence_acq_rel_gpu();
      const double bv = __longlong_as_double((long long)best_bits);
      const bool stop = !positioned && !(have && bv > p.threshold);
      if (lane == 0) {
        if (any_timeout) atomicCAS(&p.state->status, kOk, kDeviceTimeout);
        s_flag[3] = any_timeout ? 1 : 0;
        s_flag[0] = (int)best_row;
        s_flag[1] = stop ? 1 : 0;
        if (!any_timeout && !stop && cta == 0 && !positioned) p.ipiv[k] = (int)best_row;
        if (!any_timeout && stop && cta == 0) p.state->stop_k = (int)k;
      }
      if (!any_timeout && !stop) {
        // L2-only loads (ld.cg): the same slot was read four steps ago and a
        // stale L1 line must not be served.
        const int wcta = (int)((best_row - p.begin) / R);
        const double* src = xdata + ((size_t)q * p.max_ctas + wcta) * xs;
        for (int j = lane; j <= w; j += 32) prow[j] = __ldcg(src + j);
        const int pl = (int)(best_row - row0);
        if (pl >= 0 && pl < rows_here && best_row != k) {
          const double* rk = rowk + (size_t)q * xs;
          for (int j = lane; j <= w; j += 32) krow[j] = __ldcg(rk + j);
        }
      }
    }
    __syncthreads();
    if (s_flag[3]) {
      aborted = true;
      break;
    }
    if (s_flag[1]) break;  // no acceptable pivot in this column: stop at step k

    // 5-6. Swap rows k and p inside the panel, scale the multipliers, update
    // the rest of the panel, and find the next column's local candidate.
    // Each row is swapped by the thread that then updates it, so no barrier
    // separates the swap from the update.
    const long long prow_g = s_flag[0];
    const int pl = (int)(prow_g - row0);
    const bool swap_p = pl >= 0 && pl < rows_here && prow_g != k;
    const double inv = 1.0 / prow[s];
    mine = Best{0.0, -1, 0};
    const double* __restrict__ pr = prow;
    for (int r = max(0, kl) + tid; r < rows_here; r += blockDim.x) {
      double* __restrict__ row = sm + r;  // element (r, j) at row[j * RP]
      if (r == kl) {  // row k receives the pivot row; it is final from now on
        copy_row(row, pr, w, RP);
        orig[r] = (int)pr[w];
        continue;
      }
      if (swap_p && r == pl) {
        copy_row(row, krow, w, RP);
        orig[r] = (int)krow[w];
      }
      const double l = row[(size_t)s * RP] * inv;
      row[(size_t)s * RP] = l;
      if (s + 1 < w) {
        const double v = row[(size_t)(s + 1) * RP] - l * pr[s + 1];
        row[(size_t)(s + 1) * RP] = v;
        const double av = fabs(v);
        if (av > mine.val) {
          mine.val = av;
          mine.row = r;
        }
        // Remaining columns in batches of 8: all loads of a batch are
        // issued before its stores.
        int j = s + 2;
        for (; j + 8 <= w; j += 8) {
          double x[8], u[8];
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            u[b] = pr[j + b];
            x[b] = row[(size_t)(j + b) * RP];
          }
#pragma unroll
          for (int b = 0; b < 8; ++b) row[(size_t)(j + b) * RP] = x[b] - l * u[b];
        }
        for (; j < w; ++j) row[(size_t)j * RP] -= l * pr[j];
      }
    }
  }

  // The last step's swaps and updates were made by other threads than the
  // ones that write the rows back.
  __syncthreads();

  // Write the slice back.
  for (int c = 0; c < w; ++c) {
    double* dst = p.a + idx(row0, p.begin + c, p.lda);
    for (int r = tid; r < rows_here; r += blockDim.x) dst[r] = sm[(size_t)c * RP + r];
  }
  if (aborted) return;

  // Swap list: block rows [begin, end) record their source row; rows below
  // `end` that received another row append (dst, src) pairs.
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

size_t panel_smem_bytes(int w, int rows_per_cta) {
  const size_t rp = (size_t)(rows_per_cta | 1);
  return (size_t)w * rp * sizeof(double) + 2 * (size_t)(w + 1) * sizeof(double) +
         (size_t)((rows_per_cta + 3) & ~3) * sizeof(int);
}

}  // namespace dp
