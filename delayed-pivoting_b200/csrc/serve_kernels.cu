// Kernels of the small-request path of the server: solves, residuals and
// backward errors for many small factorisations at once (one CTA per item),
// on factors made by the batched factorisation (batched.cu).
//
// A factorisation P*A*Q = L*U with swap histories ipiv / jpiv (replayed in
// order, delayed_lu_cuda/example.cu:61-68) solves A x = b as
//   y = L^{-1} (P b),  y = U^{-1} y,  x = Q y,
// with (P b)[k] = b[row[k]] and x[col[k]] = y[k], row / col the histories
// replayed on the identity.
#include <algorithm>

#include "dp_device.cuh"
#include "serve_kernels.h"

namespace dp {
namespace serve {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kBlk = 32;  // diagonal block of the triangular sweeps

// Right-hand sides per pass held in shared memory.
constexpr int kChunk = 16;

__device__ __forceinline__ int ld_of(int n) { return n + 1; }

}  // namespace

// Composite row / column orders of each matrix's swap histories: one warp per
// matrix, lane 0 replaying in shared memory, the warp writing out.
__global__ void orders_kernel(const int* __restrict__ ns, const long long* __restrict__ rec,
                              const int* __restrict__ ipiv, const int* __restrict__ jpiv,
                              int* row_order, int* col_order, int count) {
  __shared__ int r[kMaxSmallN], c[kMaxSmallN];
  const int i = blockIdx.x;
  if (i >= count) return;
  const int n = ns[i];
  const long long o = rec[i];
  for (int k = threadIdx.x; k < n; k += 32) r[k] = c[k] = k;
  __syncwarp();
  if (threadIdx.x == 0)
    for (int k = 0; k < n; ++k) {
      const int p = ipiv[o + k], q = jpiv[o + k];
      const int t = r[k];
      r[k] = r[p];
      r[p] = t;
      const int u = c[k];
      c[k] = c[q];
      c[q] = u;
    }
  __syncwarp();
  for (int k = threadIdx.x; k < n; k += 32) {
    row_order[o + k] = r[k];
    col_order[o + k] = c[k];
  }
}

// X = A^{-1} B for each item.
__global__ void __launch_bounds__(kThreads) solve_kernel(const SolveItem* __restrict__ items) {
  extern __shared__ double Y[];  // [kChunk][n + 1]
  const SolveItem it = items[blockIdx.x];
  const int n = it.n, ldy = ld_of(n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* LU = it.lu;
  for (int c0 = 0; c0 < it.nrhs; c0 += kChunk) {
    const int nc = min(kChunk, it.nrhs - c0);
    __syncthreads();
    for (int e = tid; e < n * nc; e += kThreads) {
      const int i = e % n, c = e / n;
      Y[c * ldy + i] = it.B[idx(it.row[i], c0 + c, it.ldb)];
    }
    __syncthreads();
    // forward: unit lower L
    for (int kb = 0; kb < n; kb += kBlk) {
      const int kw = min(kBlk, n - kb);
      for (int c = warp; c < nc; c += kWarps) {
        double l[kBlk];
#pragma unroll
        for (int k = 0; k < kBlk; ++k)
          l[k] = (lane < kw && k < lane) ? LU[idx(kb + lane, kb + k, n)] : 0.0;
        double y = lane < kw ? Y[c * ldy + kb + lane] : 0.0;
#pragma unroll
        for (int k = 0; k < kBlk - 1; ++k) {
          const double yk = __shfl_sync(0xffffffffu, y, k);
          if (lane > k) y = fma(-l[k], yk, y);
        }
        if (lane < kw) Y[c * ldy + kb + lane] = y;
      }
      __syncthreads();
      for (int i = kb + kw + tid; i < n; i += kThreads) {
        double acc[kChunk];
#pragma unroll
        for (int c = 0; c < kChunk; ++c) acc[c] = c < nc ? Y[c * ldy + i] : 0.0;
        for (int k = 0; k < kw; ++k) {
          const double l = LU[idx(i, kb + k, n)];
#pragma unroll
          for (int c = 0; c < kChunk; ++c)
            if (c < nc) acc[c] = fma(-l, Y[c * ldy + kb + k], acc[c]);
        }
#pragma unroll
        for (int c = 0; c < kChunk; ++c)
          if (c < nc) Y[c * ldy + i] = acc[c];
      }
      __syncthreads();
    }
    // backward: upper U with its diagonal
    for (int kb = ((n - 1) / kBlk) * kBlk; kb >= 0; kb -= kBlk) {
      const int kw = min(kBlk, n - kb);
      for (int c = warp; c < nc; c += kWarps) {
        double u[kBlk];
#pragma unroll
        for (int k = 0; k < kBlk; ++k)
          u[k] = (lane < kw && k >= lane && k < kw) ? LU[idx(kb + lane, kb + k, n)] : 0.0;
        double y = lane < kw ? Y[c * ldy + kb + lane] : 0.0;
#pragma unroll
        for (int k = kBlk - 1; k >= 0; --k) {
          if (k < kw) {
            if (lane == k) y = y / u[k];
            const double yk = __shfl_sync(0xffffffffu, y, k);
            if (lane < k) y = fma(-u[k], yk, y);
          }
        }
        if (lane < kw) Y[c * ldy + kb + lane] = y;
      }
      __syncthreads();
      for (int i = tid; i < kb; i += kThreads) {
        double acc[kChunk];
#pragma unroll
        for (int c = 0; c < kChunk; ++c) acc[c] = c < nc ? Y[c * ldy + i] : 0.0;
        for (int k = 0; k < kw; ++k) {
          const double u = LU[idx(i, kb + k, n)];
#pragma unroll
          for (int c = 0; c < kChunk; ++c)
            if (c < nc) acc[c] = fma(-u, Y[c * ldy + kb + k], acc[c]);
        }
#pragma unroll
        for (int c = 0; c < kChunk; ++c)
          if (c < nc) Y[c * ldy + i] = acc[c];
      }
      __syncthreads();
    }
    for (int e = tid; e < n * nc; e += kThreads) {
      const int i = e % n, c = e / n;
      it.X[idx(it.col[i], c0 + c, it.ldx)] = Y[c * ldy + i];
    }
  }
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long*>(addr),
            (unsigned long long)__double_as_longlong(v));
}

// R = B - A X and the normwise backward error
//   max_c ||R_c||_inf / (||A||_inf ||X_c||_inf + ||B_c||_inf)
// into err[item] (NaN reported as +inf).
__global__ void __launch_bounds__(kThreads, 1) residual_kernel(const ResidualItem* __restrict__ items,
                                                            double* err) {
  extern __shared__ double Xs[];  // [kChunk][n + 1]
  __shared__ double norms[3 * kMaxRhs + 1];  // |R|, |X|, |B| per column, ||A||
  const ResidualItem it = items[blockIdx.x];
  const int n = it.n, ldx = ld_of(n), tid = threadIdx.x;
  for (int c = tid; c < 3 * kMaxRhs + 1; c += kThreads) norms[c] = 0.0;
  __syncthreads();
  // ||A||_inf: thread per row
  for (int i = tid; i < n; i += kThreads) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += fabs(it.A[idx(i, j, it.lda)]);
    atomic_max_nonneg(&norms[3 * kMaxRhs], s == s ? s : INFINITY);
  }
  for (int c0 = 0; c0 < it.nrhs; c0 += kChunk) {
    const int nc = min(kChunk, it.nrhs - c0);
    __syncthreads();
    for (int e = tid; e < n * nc; e += kThreads) {
      const int i = e % n, c = e / n;
      const double x = it.X[idx(i, c0 + c, it.ldx)];
      Xs[c * ldx + i] = x;
      const double ax = fabs(x);
      atomic_max_nonneg(&norms[kMaxRhs + c0 + c], ax == ax ? ax : INFINITY);
    }
    __syncthreads();
    for (int i = tid; i < n; i += kThreads) {
      double acc[kChunk];
#pragma unroll
      for (int c = 0; c < kChunk; ++c) acc[c] = c < nc ? it.B[idx(i, c0 + c, it.ldb)] : 0.0;
      for (int j = 0; j < n; ++j) {
        const double a = it.A[idx(i, j, it.lda)];
#pragma unroll
        for (int c = 0; c < kChunk; ++c)
          if (c < nc) acc[c] = fma(-a, Xs[c * ldx + j], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < kChunk; ++c)
        if (c < nc) {
          it.R[idx(i, c0 + c, it.ldr)] = acc[c];
          const double ar = fabs(acc[c]), ab = fabs(it.B[idx(i, c0 + c, it.ldb)]);
          atomic_max_nonneg(&norms[c0 + c], ar == ar ? ar : INFINITY);
          atomic_max_nonneg(&norms[2 * kMaxRhs + c0 + c], ab == ab ? ab : INFINITY);
        }
    }
  }
  __syncthreads();
  if (tid == 0) {
    const double na = norms[3 * kMaxRhs];
    double e = 0.0;
    for (int c = 0; c < it.nrhs; ++c) {
      const double den = na * norms[kMaxRhs + c] + norms[2 * kMaxRhs + c];
      const double v = den > 0.0 ? norms[c] / den : (norms[c] > 0.0 ? INFINITY : 0.0);
      e = fmax(e, v == v ? v : INFINITY);
    }
    err[blockIdx.x] = e;
  }
}

// X += D for each item.
__global__ void axpy_kernel(const AxpyItem* __restrict__ items) {
  const AxpyItem it = items[blockIdx.x];
  for (int e = threadIdx.x; e < it.n * it.nrhs; e += blockDim.x) {
    const int i = e % it.n, c = e / it.n;
    it.X[idx(i, c, it.ldx)] += it.D[idx(i, c, it.ldd)];
  }
}

// dst (n x m, ldd) = src (n x m, lds) for each item.
__global__ void copy_kernel(const CopyItem* __restrict__ items) {
  const CopyItem it = items[blockIdx.x];
  for (long long e = threadIdx.x; e < (long long)it.rows * it.cols; e += blockDim.x) {
    const int i = (int)(e % it.rows), c = (int)(e / it.rows);
    it.dst[idx(i, c, it.ldd)] = it.src[idx(i, c, it.lds)];
  }
}

size_t solve_smem(int max_n) { return sizeof(double) * (size_t)kChunk * (max_n + 1); }

int launch_orders(const int* ns, const long long* rec, const int* ipiv, const int* jpiv,
                  int* row_order, int* col_order, int count, cudaStream_t st) {
  if (count <= 0) return kOk;
  dp::note_launch();
  orders_kernel<<<count, 32, 0, st>>>(ns, rec, ipiv, jpiv, row_order, col_order, count);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

int launch_solve(const SolveItem* items, int count, int max_n, cudaStream_t st) {
  if (count <= 0) return kOk;
  const size_t sm = solve_smem(max_n);
  if (!ensure_smem((const void*)solve_kernel, sm)) return kCudaFailure;
  dp::note_launch();
  solve_kernel<<<count, kThreads, sm, st>>>(items);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

int launch_residual(const ResidualItem* items, double* err, int count, int max_n, cudaStream_t st) {
  if (count <= 0) return kOk;
  const size_t sm = solve_smem(max_n);
  if (!ensure_smem((const void*)residual_kernel, sm)) return kCudaFailure;
  dp::note_launch();
  residual_kernel<<<count, kThreads, sm, st>>>(items, err);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

int launch_axpy(const AxpyItem* items, int count, cudaStream_t st) {
  if (count <= 0) return kOk;
  dp::note_launch();
  axpy_kernel<<<count, kThreads, 0, st>>>(items);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

int launch_copy(const CopyItem* items, int count, cudaStream_t st) {
  if (count <= 0) return kOk;
  dp::note_launch();
  copy_kernel<<<count, kThreads, 0, st>>>(items);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

}  // namespace serve
}  // namespace dp
