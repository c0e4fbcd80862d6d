// Multifrontal hand-off (no reference code; the reference's design document
// describes it, doc/（非）对称稠密矩阵的延迟主元LU方法.md:228-457): a frontal
// matrix F (m x n) whose leading p rows and p columns are fully summed is
// factored partially - pivots only inside the fully-summed block, with the
// delayed-pivoting rules of delayed_lu/delayed_dgetrf.cpp:129-251 - and what
// is left, the Schur complement of the k eliminated pivots over the whole
// front (the delayed rows and columns of the fully-summed block first), is the
// contribution block handed to the parent front, where extend-add scatters it
// through the two fronts' global index lists.
//
// Steps (all on the device, the records of the fully-summed block on the
// host as for every dp_getrf_* call):
//   1. F11 = F(0:p, 0:p) by the delayed LU (k = its info, records ipiv/jpiv);
//   2. its composite row / column permutation applied to F12 = F(0:p, p:n)
//      and F21 = F(p:m, 0:p);
//   3. U12 = L11^{-1} F12(0:k, :), F12(k:p, :) -= L(k:p, 0:k) U12;
//   4. L21 = F21(:, 0:k) U11^{-1} (right-side solve, 32-column blocks: the
//      block's solve per row, then a DMMA update of the columns after it),
//      F21(:, k:p) -= L21 U(0:k, k:p);
//   5. F22 -= L21 U12.
#include <algorithm>
#include <vector>

#include "delayed_pivoting_b200.h"
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {
namespace front {
namespace {

constexpr int kThreads = 256;
constexpr int kSolveW = 32;  // columns of one right-side solve block

// out(i, c) = a(src[i], c) for i < rows, c < cols (a row gather).
__global__ void gather_rows_kernel(const double* __restrict__ a, long long lda, int rows, int cols,
                                   const int* __restrict__ src, double* __restrict__ out,
                                   long long ldo) {
  const long long total = (long long)rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % rows), c = (int)(e / rows);
    out[idx(i, c, ldo)] = a[idx(src[i], c, lda)];
  }
}

// out(i, c) = a(i, src[c]) for i < rows, c < cols (a column gather).
__global__ void gather_cols_kernel(const double* __restrict__ a, long long lda, int rows, int cols,
                                   const int* __restrict__ src, double* __restrict__ out,
                                   long long ldo) {
  const long long total = (long long)rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % rows), c = (int)(e / rows);
    out[idx(i, c, ldo)] = a[idx(i, src[c], lda)];
  }
}

// X = B U^{-1} for the rows x w block B (w <= kSolveW), U upper with its
// diagonal (w x w): one thread per row, the row in registers, U staged in
// shared memory; x_j = (b_j - sum_{i<j} x_i u_ij) * (1 / u_jj), the sum in
// order i = 0, 1, ... as the right-looking elimination forms it.
__global__ void __launch_bounds__(kThreads)
rsolve_upper_kernel(double* __restrict__ B, long long ldb, int rows, int w,
                    const double* __restrict__ U, long long ldu) {
  __shared__ double us[kSolveW * kSolveW];  // us[j * kSolveW + i] = U(i, j), i <= j
  __shared__ double rinv[kSolveW];
  for (int e = threadIdx.x; e < kSolveW * kSolveW; e += blockDim.x) {
    const int j = e / kSolveW, i = e - j * kSolveW;
    us[e] = (i <= j && j < w) ? U[idx(i, j, ldu)] : 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < w; j += blockDim.x) rinv[j] = 1.0 / us[j * kSolveW + j];
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  double x[kSolveW];
#pragma unroll
  for (int j = 0; j < kSolveW; ++j) x[j] = j < w ? B[idx(r, j, ldb)] : 0.0;
#pragma unroll
  for (int j = 0; j < kSolveW; ++j) {
    if (j >= w) break;
#pragma unroll
    for (int i = 0; i < j; ++i) x[j] = fma(-x[i], us[j * kSolveW + i], x[j]);
    x[j] *= rinv[j];
  }
#pragma unroll
  for (int j = 0; j < kSolveW; ++j)
    if (j < w) B[idx(r, j, ldb)] = x[j];
}

// P(prow[i], pcol[j]) += C(i, j): one thread per element, consecutive
// threads on consecutive rows of C.
__global__ void extend_add_kernel(int mc, int nc, const double* __restrict__ C, long long ldc,
                                  const int* __restrict__ prow, const int* __restrict__ pcol,
                                  double* __restrict__ P, long long ldp) {
  const long long total = (long long)mc * nc;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % mc), j = (int)(e / mc);
    P[idx(prow[i], pcol[j], ldp)] += C[idx(i, j, ldc)];
  }
}

int grid_of(long long work) {
  return (int)std::max(1LL, std::min<long long>((work + kThreads - 1) / kThreads, 148LL * 16));
}

// Composite permutation of a swap history: src[i] = the row whose content
// position i holds after swaps (k, rec[k]) for k = 0, 1, ..., count - 1.
std::vector<int> composite(const int* rec, int count, int size) {
  std::vector<int> src(size);
  for (int i = 0; i < size; ++i) src[i] = i;
  for (int k = 0; k < count; ++k) std::swap(src[k], src[rec[k]]);
  return src;
}

}  // namespace
}  // namespace front

// Right-side solve X = B U^{-1} for B rows x w (column-major, ldb) and U the
// w x w upper triangle at u (ldu): 32-column blocks, each solved per row and
// then subtracted from the columns after it by the DMMA update.
void rsolve_upper(double* B, long long ldb, int rows, int w, const double* U, long long ldu,
                  cudaStream_t st) {
  if (rows <= 0 || w <= 0) return;
  for (int j0 = 0; j0 < w; j0 += front::kSolveW) {
    const int wb = std::min(front::kSolveW, w - j0);
    dp::note_launch();
    front::rsolve_upper_kernel<<<(rows + front::kThreads - 1) / front::kThreads, front::kThreads,
                                 0, st>>>(B + idx(0, j0, ldb), ldb, rows, wb,
                                          U + idx(j0, j0, ldu), ldu);
    if (j0 + wb < w)
      launch_gemm_minus(rows, w - j0 - wb, wb, B + idx(0, j0, ldb), ldb,
                        U + idx(j0, j0 + wb, ldu), ldu, B + idx(0, j0 + wb, ldb), ldb, st);
  }
}

}  // namespace dp

namespace dp {

int getrf_device(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                 cudaStream_t st, const dp_options* opt);

namespace front {

// Steps 2-5 of the hand-off after F11 is factored (k pivots, records ip / jp
// of the p fully-summed rows / columns).  `tmp` holds max(p (n - p),
// (m - p) p) doubles; `d_src` p ints.
int finish(int m, int n, int p, int k, double* F, long long ldf, const int* ip, const int* jp,
           double* tmp, int* d_src, cudaStream_t st) {
  const int mr = m - p, nr = n - p;
  // 2. the fully-summed block's row order on F12, column order on F21
  if (nr > 0) {
    const std::vector<int> rsrc = composite(ip, p, p);
    if (cudaMemcpyAsync(d_src, rsrc.data(), sizeof(int) * p, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      return kCudaFailure;
    note_launch();
    gather_rows_kernel<<<grid_of((long long)p * nr), kThreads, 0, st>>>(F + idx(0, p, ldf), ldf, p,
                                                                        nr, d_src, tmp, p);
    launch_copy_block(tmp, p, F + idx(0, p, ldf), ldf, p, nr, st);
  }
  if (mr > 0) {
    const std::vector<int> csrc = composite(jp, p, p);
    if (cudaMemcpyAsync(d_src, csrc.data(), sizeof(int) * p, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      return kCudaFailure;
    note_launch();
    gather_cols_kernel<<<grid_of((long long)mr * p), kThreads, 0, st>>>(F + idx(p, 0, ldf), ldf, mr,
                                                                        p, d_src, tmp, mr);
    launch_copy_block(tmp, mr, F + idx(p, 0, ldf), ldf, mr, p, st);
  }
  if (k > 0) {
    // 3. U12 = L11^{-1} F12 in 64-row blocks, then the delayed rows of F12
    if (nr > 0) {
      const int tw = trsm_max_width();
      for (int b = 0; b < k; b += tw) {
        const int wb = std::min(tw, k - b);
        launch_trsm_unit_lower(F, ldf, b, wb, p, nr, st);
        if (b + wb < p)  // rows after the block: the rest of U12 and the delayed rows
          launch_gemm_minus(p - b - wb, nr, wb, F + idx(b + wb, b, ldf), ldf, F + idx(b, p, ldf),
                            ldf, F + idx(b + wb, p, ldf), ldf, st);
      }
    }
    if (mr > 0) {
      // 4. L21 = F21 U11^{-1}, then the delayed columns of F21
      rsolve_upper(F + idx(p, 0, ldf), ldf, mr, k, F, ldf, st);
      if (p > k)
        launch_gemm_minus(mr, p - k, k, F + idx(p, 0, ldf), ldf, F + idx(0, k, ldf), ldf,
                          F + idx(p, k, ldf), ldf, st);
      // 5. the rest of the front
      if (nr > 0)
        launch_gemm_minus(mr, nr, k, F + idx(p, 0, ldf), ldf, F + idx(0, p, ldf), ldf,
                          F + idx(p, p, ldf), ldf, st);
    }
  }
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

}  // namespace front
}  // namespace dp

extern "C" {

int dp_front_factor(int m, int n, int p, double* d_f, int ldf, int* row_index, int* col_index,
                    int* ipiv, int* jpiv, int* npiv, void* stream) {
  if (npiv) *npiv = -1;
  if (m < 0 || n < 0 || p < 0 || p > std::min(m, n) || ldf < std::max(1, m) || !npiv ||
      (m > 0 && n > 0 && !d_f) || (p > 0 && (!ipiv || !jpiv)))
    return dp::kInvalidArgument;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int k = 0;
  if (p > 0) {
    // 1. the fully-summed block alone: pivots only among its rows and columns
    const int s = dp::getrf_device(p, p, d_f, ldf, ipiv, jpiv, &k, st, nullptr);
    if (s != dp::kOk) return s;
  }
  const size_t tmp_doubles =
      std::max((size_t)p * (size_t)(n - p), (size_t)(m - p) * (size_t)p);
  double* tmp = nullptr;
  int* d_src = nullptr;
  int status = dp::kOk;
  if (p > 0 && tmp_doubles > 0) {
    if (cudaMallocAsync(reinterpret_cast<void**>(&tmp), sizeof(double) * tmp_doubles, st) !=
            cudaSuccess ||
        cudaMallocAsync(reinterpret_cast<void**>(&d_src), sizeof(int) * (size_t)p, st) !=
            cudaSuccess) {
      cudaGetLastError();
      status = dp::kAllocationFailed;
    }
    if (status == dp::kOk)
      status = dp::front::finish(m, n, p, k, d_f, ldf, ipiv, jpiv, tmp, d_src, st);
  }
  if (tmp) cudaFreeAsync(tmp, st);
  if (d_src) cudaFreeAsync(d_src, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && status == dp::kOk) status = dp::kCudaFailure;
  if (status != dp::kOk) {
    cudaGetLastError();
    return status;
  }
  // the global index lists follow the fully-summed block's permutations
  if (row_index && p > 0) {
    const std::vector<int> src = dp::front::composite(ipiv, p, p);
    std::vector<int> old(row_index, row_index + p);
    for (int i = 0; i < p; ++i) row_index[i] = old[src[i]];
  }
  if (col_index && p > 0) {
    const std::vector<int> src = dp::front::composite(jpiv, p, p);
    std::vector<int> old(col_index, col_index + p);
    for (int i = 0; i < p; ++i) col_index[i] = old[src[i]];
  }
  *npiv = k;
  return dp::kOk;
}

int dp_extend_add(int mc, int nc, const double* d_c, int ldc, const int* d_prow, const int* d_pcol,
                  double* d_p, int ldp, void* stream) {
  if (mc < 0 || nc < 0 || ldc < std::max(1, mc) || ldp < 1) return dp::kInvalidArgument;
  if (mc == 0 || nc == 0) return dp::kOk;
  if (!d_c || !d_prow || !d_pcol || !d_p) return dp::kInvalidArgument;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dp::note_launch();
  dp::front::extend_add_kernel<<<dp::front::grid_of((long long)mc * nc), dp::front::kThreads, 0,
                                 st>>>(mc, nc, d_c, ldc, d_prow, d_pcol, d_p, ldp);
  return cudaGetLastError() == cudaSuccess ? dp::kOk : dp::kCudaFailure;
}

}  // extern "C"
