// Row and column permutation kernels of the delayed-pivoting LU.
//
// The reference swaps a full row (n elements, stride lda) and, on a fallback,
// a full column (m elements) at every step (delayed_lu/delayed_dgetrf.cpp:202-209,
// delayed_lu_cuda/delayed_dgetrf_cuda.cu:304-317).  Here the panel kernel
// swaps rows only inside the panel columns and writes the composite
// permutation of the whole panel as a list of (destination, source) rows;
// laswp_kernel then moves, per column outside the panel, only the rows that
// changed, once per panel: each warp owns one column, gathers every source
// row into registers and scatters them to their destinations.  The block
// part of the list (destinations begin..end-1) is contiguous, so those writes
// are coalesced.  Full-row / full-column swaps of a fallback step are
// separate grid-stride kernels.
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int kLaswpThreads = 256;
constexpr int kMaxSwapEntries = 512;  // 2 * maximum panel width
constexpr int kPerLane = kMaxSwapEntries / 32;
constexpr int kSolveW = 64;           // widest panel whose block rows laswp_kernel solves

// Also, for the columns [s0, s1) (a subset of [c2, c3)) and a panel of at most
// kSolveW columns that did not stop (state->stop_k < 0): U12 = L11^{-1} of the
// panel's block rows right after they are permuted, L11 the panel's unit
// lower triangle (the in-block TRSM, delayed_lu/delayed_dgetrf.cpp:72-74,
// fused: one warp per column, rows begin + lane and begin + 32 + lane, the
// entries of step k passed by shuffle, the same order of operations per row
// as the TRSM kernel).
__global__ void __launch_bounds__(kLaswpThreads)
laswp_kernel(double* a, long long lda, int begin, int nblock, const int* swap_block,
             const int* swap_extra, const State* state, int c0, int c1, int c2, int c3,
             int gate_begin, int s0, int s1) {
  __shared__ int s_dst[kMaxSwapEntries];
  __shared__ int s_src[kMaxSwapEntries];
  __shared__ int s_count;
  __shared__ double s_l[kSolveW * kSolveW];  // s_l[k * kSolveW + i] = L11(i, k), i > k
  const int sk = state->stop_k;
  if (gate_begin >= 0 && sk >= 0 && sk < gate_begin) return;  // an earlier panel stopped
  const bool solve = s0 < s1 && sk < 0 && nblock <= kSolveW;
  const int tid = threadIdx.x;
  if (solve) {
    for (int e = tid; e < kSolveW * kSolveW; e += blockDim.x) {
      const int k = e / kSolveW, i = e - k * kSolveW;
      s_l[e] = (i > k && i < nblock) ? a[idx(begin + i, begin + k, lda)] : 0.0;
    }
  }
  const int nextra = min(state->swap_count, kMaxSwapEntries - nblock);
  if (tid == 0) s_count = 0;
  __syncthreads();
  // keep only rows whose content changed (warp-aggregated compaction)
  for (int base = 0; base < nblock + nextra; base += blockDim.x) {
    const int i = base + tid;
    int d = 0, sr = 0;
    bool keep = false;
    if (i < nblock) {
      d = begin + i;
      sr = swap_block[i];
      keep = sr != d;
    } else if (i < nblock + nextra) {
      d = swap_extra[2 * (i - nblock)];
      sr = swap_extra[2 * (i - nblock) + 1];
      keep = sr != d;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    int wbase = 0;
    if ((tid & 31) == 0 && mask) wbase = atomicAdd(&s_count, __popc(mask));
    wbase = __shfl_sync(0xffffffffu, wbase, 0);
    if (keep) {
      const int pos = wbase + __popc(mask & ((1u << (tid & 31)) - 1u));
      s_dst[pos] = d;
      s_src[pos] = sr;
    }
    __syncthreads();
  }
  __syncthreads();
  const int total = s_count;
  if (total == 0 && !solve) return;

  const int lane = tid & 31;
  const int warps = blockDim.x >> 5;
  const long long n1 = c1 - c0, ncols = n1 + (c3 - c2);
  for (long long cid = (long long)blockIdx.x * warps + (tid >> 5); cid < ncols;
       cid += (long long)gridDim.x * warps) {
    const long long col = cid < n1 ? c0 + cid : c2 + (cid - n1);
    double* ac = a + idx(0, col, lda);
    double v[kPerLane];
#pragma unroll
    for (int j = 0; j < kPerLane; ++j) {
      const int i = lane + 32 * j;
      if (i < total) v[j] = ac[s_src[i]];
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kPerLane; ++j) {
      const int i = lane + 32 * j;
      if (i < total) ac[s_dst[i]] = v[j];
    }
    __syncwarp();
    if (solve && col >= s0 && col < s1) {  // (warp-uniform)
      double* bc = ac + begin;
      double x0 = lane < nblock ? bc[lane] : 0.0;
      double x1 = 32 + lane < nblock ? bc[32 + lane] : 0.0;
      for (int k = 0; k < nblock - 1; ++k) {
        const double xk = __shfl_sync(0xffffffffu, k < 32 ? x0 : x1, k & 31);
        // only rows below k (an infinite or NaN x_k must not reach the others)
        if (lane > k) x0 = fma(-s_l[k * kSolveW + lane], xk, x0);
        if (32 + lane > k) x1 = fma(-s_l[k * kSolveW + 32 + lane], xk, x1);
      }
      if (lane < nblock) bc[lane] = x0;
      if (32 + lane < nblock) bc[32 + lane] = x1;
      __syncwarp();
    }
  }
}

// The swap lists of consecutive panels applied in panel order: list p covers
// the panel starting at row begin_p = q.base + width[0] + ... + width[p-1],
// its block part at blk[begin_p - q.base] and up to width[p] extra pairs at
// ext[2 (begin_p - q.base)] (unused pairs have a negative destination: the
// region is filled with -1 before the panel runs, and the panel writes its
// pairs from the front).  Each CTA compacts every list into shared memory
// (list p at [s_lb[p], s_lb[p+1])); each warp then applies the lists to one
// column in turn, gathering a list's sources before scattering it, so the
// result equals launching laswp_kernel once per panel.
__global__ void __launch_bounds__(kLaswpThreads)
laswp_seq_kernel(double* a, long long lda, const int* blk, const int* ext, SwapSeq q, int c0,
                 int c1, int c2, int c3) {
  __shared__ int s_dst[kSwapSeqEntries];
  __shared__ int s_src[kSwapSeqEntries];
  __shared__ int s_lb[kSwapSeqLists + 1];
  __shared__ int s_count;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_count = 0;
    s_lb[0] = 0;
  }
  __syncthreads();
  int off = 0;
  for (int p = 0; p < q.lists; ++p) {
    const int nblock = q.width[p], nextra = q.width[p];
    for (int base = 0; base < nblock + nextra; base += blockDim.x) {
      const int i = base + tid;
      int d = 0, sr = 0;
      bool keep = false;
      if (i < nblock) {
        d = q.base + off + i;
        sr = blk[off + i];
        keep = sr != d;
      } else if (i < nblock + nextra) {
        d = ext[2 * off + 2 * (i - nblock)];
        sr = ext[2 * off + 2 * (i - nblock) + 1];
        keep = d >= 0 && sr != d;
      }
      const unsigned mask = __ballot_sync(0xffffffffu, keep);
      int wbase = 0;
      if ((tid & 31) == 0 && mask) wbase = atomicAdd(&s_count, __popc(mask));
      wbase = __shfl_sync(0xffffffffu, wbase, 0);
      if (keep) {
        const int pos = wbase + __popc(mask & ((1u << (tid & 31)) - 1u));
        s_dst[pos] = d;
        s_src[pos] = sr;
      }
      __syncthreads();
    }
    // the list's last append is behind the barrier above; no thread appends
    // to the next list before the boundary is read
    if (tid == 0) s_lb[p + 1] = s_count;
    __syncthreads();
    off += nblock;
  }
  if (s_count == 0) return;

  const int lane = tid & 31;
  const int warps = blockDim.x >> 5;
  const long long n1 = c1 - c0, ncols = n1 + (c3 - c2);
  for (long long cid = (long long)blockIdx.x * warps + (tid >> 5); cid < ncols;
       cid += (long long)gridDim.x * warps) {
    const long long col = cid < n1 ? c0 + cid : c2 + (cid - n1);
    double* ac = a + idx(0, col, lda);
    for (int p = 0; p < q.lists; ++p) {
      const int lo = s_lb[p], cnt = s_lb[p + 1] - lo;
      if (cnt == 0) continue;
      double v[kPerLane];
#pragma unroll
      for (int j = 0; j < kPerLane; ++j) {
        const int i = lane + 32 * j;
        if (i < cnt) v[j] = ac[s_src[lo + i]];
      }
      __syncwarp();
#pragma unroll
      for (int j = 0; j < kPerLane; ++j) {
        const int i = lane + 32 * j;
        if (i < cnt) ac[s_dst[lo + i]] = v[j];
      }
      __syncwarp();
    }
  }
}

__global__ void swap_row_kernel(double* a, long long lda, int n, int r1, int r2) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const double t = a[idx(r1, j, lda)];
    a[idx(r1, j, lda)] = a[idx(r2, j, lda)];
    a[idx(r2, j, lda)] = t;
  }
}

__global__ void swap_col_kernel(double* a, long long lda, int m, int c1, int c2) {
  double* x = a + idx(0, c1, lda);
  double* y = a + idx(0, c2, lda);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    const double t = x[i];
    x[i] = y[i];
    y[i] = t;
  }
}

__global__ void identity_records_kernel(int* ipiv, int* jpiv, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    ipiv[i] = i;
    jpiv[i] = i;
  }
}

__global__ void set_record_kernel(int* ipiv, int* jpiv, int k, int p, int q) {
  ipiv[k] = p;
  jpiv[k] = q;
}

int grid_for(long long work, int threads, int cap) {
  long long g = (work + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

}  // namespace

void launch_laswp(double* a, long long lda, int begin, int nblock, const int* swap_block,
                  const int* swap_extra, const State* state, int c0, int c1, int c2, int c3,
                  cudaStream_t s, int gate_begin, int s0, int s1) {
  const long long ncols = (long long)(c1 - c0) + (c3 - c2);
  if (ncols <= 0 || nblock <= 0) return;
  const int warps = kLaswpThreads / 32;
  const int grid = grid_for(ncols, warps, 148 * 16);
  dp::note_launch();
  laswp_kernel<<<grid, kLaswpThreads, 0, s>>>(a, lda, begin, nblock, swap_block, swap_extra,
                                              state, c0, c1, c2, c3, gate_begin, s0, s1);
}

int laswp_solve_max_width() { return kSolveW; }

int launch_laswp_seq(double* a, long long lda, const int* blk, const int* ext, int base,
                     const int* widths, int lists, int c0, int c1, int c2, int c3,
                     cudaStream_t s) {
  const long long ncols = (long long)(c1 - c0) + (c3 - c2);
  if (ncols <= 0 || lists <= 0) return 0;
  for (int i = 0; i < lists; ++i)  // a panel list: at most kMaxSwapEntries changed rows
    if (widths[i] < 1 || 2 * widths[i] > kMaxSwapEntries) return -1;
  const int warps = kLaswpThreads / 32;
  const int grid = grid_for(ncols, warps, 148 * 16);
  int launches = 0, p = 0, off = 0;
  while (p < lists) {
    // as many whole lists as fit the kernel's list and entry capacity
    SwapSeq q;
    q.base = base + off;
    q.lists = 0;
    int entries = 0, width = 0;
    while (p < lists && q.lists < kSwapSeqLists && entries + 2 * widths[p] <= kSwapSeqEntries) {
      q.width[q.lists] = widths[p];
      entries += 2 * widths[p];
      width += widths[p];
      ++q.lists;
      ++p;
    }
    if (q.lists == 0) return -1;  // one list beyond the capacity: not a panel's list
    dp::note_launch();
    laswp_seq_kernel<<<grid, kLaswpThreads, 0, s>>>(a, lda, blk + off, ext + 2 * off, q, c0, c1,
                                                    c2, c3);
    ++launches;
    off += width;
  }
  return launches;
}

void launch_swap_row(double* a, long long lda, int n, int r1, int r2, cudaStream_t s) {
  if (r1 == r2 || n <= 0) return;
  dp::note_launch();
  swap_row_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(a, lda, n, r1, r2);
}

void launch_swap_col(double* a, long long lda, int m, int c1, int c2, cudaStream_t s) {
  if (c1 == c2 || m <= 0) return;
  dp::note_launch();
  swap_col_kernel<<<grid_for(m, 256, 148 * 8), 256, 0, s>>>(a, lda, m, c1, c2);
}

void launch_set_record(int* ipiv, int* jpiv, int k, int p, int q, cudaStream_t s) {
  dp::note_launch();
  set_record_kernel<<<1, 1, 0, s>>>(ipiv, jpiv, k, p, q);
}

void launch_identity_records(int* ipiv, int* jpiv, int count, cudaStream_t s) {
  if (count <= 0) return;
  dp::note_launch();
  identity_records_kernel<<<grid_for(count, 256, 148 * 4), 256, 0, s>>>(ipiv, jpiv, count);
}

}  // namespace dp
