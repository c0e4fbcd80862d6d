// Kernels of the server's small-request path (serve_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "delayed_pivoting_b200.h"

namespace dp {
namespace batch {
// Bytes of the scratch `d_queue` of launch_raw: the work counter and the
// launch's near-tie counters (decisions checked, order-sensitive decisions,
// largest runner-up / winner ratio as bits) at byte 8.
constexpr size_t kQueueBytes = 32;
// The batched factorisation on caller-managed device arrays (batched.cu).
int launch_raw(int count, int max_n, int sms, const int* d_n, const long long* d_off,
               const long long* d_rec, const int* d_order, int* d_queue, double* base, int* ipiv,
               int* jpiv, int* info, const dp_batch_options& opt, cudaStream_t st);
}  // namespace batch


namespace serve {

constexpr int kMaxSmallN = 512;  // largest order on the small path (the batched kernel's)
constexpr int kMaxRhs = 64;      // right-hand sides per solve item

struct SolveItem {   // X = A^{-1} B through factors P A Q = L U
  const double* lu;  // n x n compact L\U, lda n
  const int* row;    // row order: (P b)[k] = b[row[k]]
  const int* col;    // column order: x[col[k]] = y[k]
  const double* B;
  double* X;
  int n, nrhs, ldb, ldx;
};

struct ResidualItem {  // R = B - A X, backward error of X
  const double* A;
  const double* B;
  const double* X;
  double* R;
  int n, nrhs, lda, ldb, ldx, ldr;
};

struct AxpyItem {  // X += D
  double* X;
  const double* D;
  int n, nrhs, ldx, ldd;
};

struct CopyItem {  // dst = src (rows x cols)
  double* dst;
  const double* src;
  int rows, cols, ldd, lds;
};

size_t solve_smem(int max_n);
int launch_orders(const int* ns, const long long* rec, const int* ipiv, const int* jpiv,
                  int* row_order, int* col_order, int count, cudaStream_t st);
int launch_solve(const SolveItem* items, int count, int max_n, cudaStream_t st);
int launch_residual(const ResidualItem* items, double* err, int count, int max_n, cudaStream_t st);
int launch_axpy(const AxpyItem* items, int count, cudaStream_t st);
int launch_copy(const CopyItem* items, int count, cudaStream_t st);

}  // namespace serve
}  // namespace dp
