// Fallback pivot searches over the active submatrix A(k:m, k:n), run only
// when the current column has no acceptable pivot.
//
// search_active_kernel: full-pivot argmax (delayed_lu/delayed_dgetrf.cpp:32-47,
//   delayed_lu_cuda/delayed_dgetrf_cuda.cu:24-85): larger magnitude wins,
//   ties go to the smaller column and then the smaller row, NaN never wins.
//   One warp per column, lanes read the column coalesced; per-block
//   candidates are reduced by the last block to finish (no second launch, no
//   host round trip for the reduction).
// search_nonzero_column_kernel: the column-fallback policy
//   (delayed_lu/delayed_dgetrf_column.cpp:30-45): the right-most column
//   j in (k, n) whose active part holds a magnitude above the threshold, with
//   that column's argmax row.
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int kSearchThreads = 256;

// Lane 0 gets the warp's best candidate and runner-up.
__device__ __forceinline__ Cand warp_best_cand(Cand v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    Cand o;
    o.val = __shfl_down_sync(0xffffffffu, v.val, off);
    o.row = __shfl_down_sync(0xffffffffu, v.row, off);
    o.col = __shfl_down_sync(0xffffffffu, v.col, off);
    o.sec = __shfl_down_sync(0xffffffffu, v.sec, off);
    v = cand_merge(v, o);
  }
  return v;
}

__device__ Cand block_best(Cand v, Cand* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_best_cand(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    Cand x = lane < (int)(blockDim.x >> 5) ? red[lane] : Cand{0.0, 0x7fffffff, 0x7fffffff, 0.0};
    x = warp_best_cand(x);
    if (lane == 0) red[0] = x;
  }
  __syncthreads();
  return red[0];
}

__global__ void __launch_bounds__(kSearchThreads)
search_active_kernel(const double* a, long long lda, int m, int n, int k, State* state,
                     Cand* block_cands) {
  __shared__ Cand red[kSearchThreads / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31;
  const long long warps_total = (long long)gridDim.x * (blockDim.x >> 5);
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  // Start from (0, k, k): a zero or NaN never replaces it, so an all-zero
  // active block reports magnitude 0 at (k, k).
  Cand best{0.0, k, k, 0.0};
  for (long long j = k + gw; j < n; j += warps_total) {
    const double* col = a + idx(0, j, lda);
    for (long long r = k + lane; r < m; r += 32) {
      const double v = fabs(col[r]);
      const Cand c{v, (int)r, (int)j, 0.0};
      best = cand_merge(best, c);
    }
  }
  best = block_best(best, red);
  if (threadIdx.x == 0) {
    block_cands[blockIdx.x] = best;
    __threadfence();
    const unsigned done = atomicAdd(&state->search_done, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  Cand v{0.0, k, k, 0.0};
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v = cand_merge(v, block_cands[i]);
  v = block_best(v, red);
  if (threadIdx.x == 0) {
    state->fallback = v;
    state->search_done = 0;
    note_decision(state, k, v.val, v.sec);
  }
}

// Grid-stride over columns j in (k, n); each warp finds its column's argmax
// and raises best column with atomicMax when the magnitude passes the
// threshold.  The last block then scans the winning column for its argmax row.
__global__ void __launch_bounds__(kSearchThreads)
search_nonzero_column_kernel(const double* a, long long lda, int m, int n, int k,
                             double threshold, State* state) {
  __shared__ Cand red[kSearchThreads / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31;
  const long long warps_total = (long long)gridDim.x * (blockDim.x >> 5);
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (long long j = k + 1 + gw; j < n; j += warps_total) {
    const double* col = a + idx(0, j, lda);
    double mx = 0.0;
    for (long long r = k + lane; r < m; r += 32) {
      const double v = fabs(col[r]);
      if (v > mx) mx = v;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    if (lane == 0 && mx > threshold) atomicMax(&state->fallback.col, (int)j);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&state->search_done, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int j = *(volatile int*)&state->fallback.col;
  Cand v{0.0, k, k, 0.0};
  if (j > k) {
    const double* col = a + idx(0, j, lda);
    for (long long r = k + threadIdx.x; r < m; r += blockDim.x)
      v = cand_merge(v, Cand{fabs(col[r]), (int)r, j, 0.0});
  }
  v = block_best(v, red);
  if (threadIdx.x == 0) {
    if (j <= k) v = Cand{0.0, k, k, 0.0};
    state->fallback = v;
    state->search_done = 0;
    // the column is chosen exactly (nonzero or not); its row is an argmax
    note_decision(state, k, v.val, v.sec);
  }
}

__global__ void reset_fallback_kernel(State* state, int k) {
  state->fallback = Cand{0.0, k, -1, 0.0};
  state->search_done = 0;
}

}  // namespace

void launch_search_active(const double* a, long long lda, int m, int n, int k, State* state,
                          Cand* block_cands, int max_blocks, cudaStream_t s) {
  const long long cols = (long long)n - k;
  const int warps = kSearchThreads / 32;
  long long grid = (cols + warps - 1) / warps;
  if (grid > max_blocks) grid = max_blocks;
  if (grid < 1) grid = 1;
  dp::note_launch();
  search_active_kernel<<<(int)grid, kSearchThreads, 0, s>>>(a, lda, m, n, k, state, block_cands);
}

void launch_search_nonzero_column(const double* a, long long lda, int m, int n, int k,
                                  double threshold, State* state, cudaStream_t s) {
  dp::note_launch();
  reset_fallback_kernel<<<1, 1, 0, s>>>(state, k);
  const long long cols = (long long)n - k - 1;
  const int warps = kSearchThreads / 32;
  long long grid = (cols + warps - 1) / warps;
  if (grid > 148 * 8) grid = 148 * 8;
  if (grid < 1) grid = 1;
  dp::note_launch();
  search_nonzero_column_kernel<<<(int)grid, kSearchThreads, 0, s>>>(a, lda, m, n, k, threshold,
                                                                   state);
}

}  // namespace dp
