// Solve and iterative refinement on top of the delayed-pivoting LU.
//
// The reference stops at the factorisation (no getrs, no refinement).  The
// factorisation P*A*Q = L*U it produces (delayed_lu_cuda/delayed_dgetrf_cuda.hpp:15-21:
// ipiv / jpiv are swap histories replayed in order, example.cu:61-68) gives
//   A x = b  <=>  L U y = P b,  x = Q y.
// getrs: gather b through the row order of ipiv, forward substitution with
// the unit-lower L and back substitution with U (64-row diagonal blocks on
// the TRSM kernels, the off-diagonal blocks as FP64 DMMA GEMM updates),
// scatter y through the column order of jpiv.
// gesv_ir: factor (mixed precision: BF16x3 tensor-core trailing update, or
// plain FP64), solve, then refine in FP64: r = b - A x on the FP64 GEMM,
// backward error max_c ||r_c||_inf / (||A||_inf ||x_c||_inf + ||b_c||_inf),
// correction through the same factors.  A refinement that stops improving
// (error not halved) or does not reach the tolerance within max_iter steps
// triggers a plain FP64 re-factorisation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "delayed_pivoting_b200.h"
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

int getrf_device(int m, int n, double* d_a, int lda, int* ipiv, int* jpiv, int* info,
                 cudaStream_t st, const dp_options* opt);

namespace {

__global__ void gather_rows_kernel(const double* __restrict__ in, long long ldi, double* out,
                                   long long ldo, const int* __restrict__ perm, int n, int nrhs) {
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    out[idx(i, c, ldo)] = in[idx(perm[i], c, ldi)];
  }
}

__global__ void scatter_rows_kernel(const double* __restrict__ in, long long ldi, double* out,
                                    long long ldo, const int* __restrict__ perm, int n, int nrhs) {
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    out[idx(perm[i], c, ldo)] = in[idx(i, c, ldi)];
  }
}

__global__ void copy_kernel(const double* __restrict__ in, long long ldi, double* out, long long ldo,
                            int n, int nrhs) {
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    out[idx(i, c, ldo)] = in[idx(i, c, ldi)];
  }
}

__global__ void axpy_kernel(const double* __restrict__ d, long long ldd, double* x, long long ldx,
                            int n, int nrhs) {
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    x[idx(i, c, ldx)] += d[idx(i, c, ldd)];
  }
}

__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// Largest max |u_ii| / min |u_ii| of mixed-precision factors kept for
// refinement (see factor_create).
constexpr double kMixedPivotRatio = 1e8;

// out[0] = max_i |D(i, i)|, out[1] = min_i |D(i, i)| of the n x n matrix D
// (out[0] zero and out[1] +inf on entry; NaN reported as +inf in both).
__global__ void diag_range_kernel(const double* __restrict__ D, long long ldd, int n, double* out) {
  double hi = 0.0, lo = __longlong_as_double(0x7ff0000000000000ll);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = fabs(D[idx(i, i, ldd)]);
    hi = (v == v) ? fmax(hi, v) : __longlong_as_double(0x7ff0000000000000ll);
    lo = (v == v) ? fmin(lo, v) : lo;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, off));
    lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(out, hi);
    atomicMin(reinterpret_cast<unsigned long long*>(out + 1),
              (unsigned long long)__double_as_longlong(lo));
  }
}

// out[c] = max_i |X(i, c)| (out must be zero on entry); NaN is reported as +inf.
__global__ void colmax_kernel(const double* __restrict__ X, long long ldx, int n, int nrhs,
                              double* out) {
  const int c = blockIdx.y;
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = fabs(X[idx(i, c, ldx)]);
    m = (v == v) ? fmax(m, v) : __longlong_as_double(0x7ff0000000000000ll);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomic_max_pos(out + c, m);
}

// rowsum[i] = sum_j |A(i, j)| over the n x n matrix (threads over rows, so
// each column is read coalesced); out[0] = max_i rowsum (atomic).
__global__ void row_abs_sum_kernel(const double* __restrict__ A, long long lda, int n, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (i < n)
    for (int j = 0; j < n; ++j) s += fabs(A[idx(i, j, lda)]);
  if (i < n) atomic_max_pos(out, s == s ? s : __longlong_as_double(0x7ff0000000000000ll));
}

// out (n x n, leading dimension n) = in^T.  32 x 32 tiles through shared
// memory (padded), both sides coalesced.
__global__ void transpose_kernel(const double* __restrict__ in, long long ldi, double* out, int n) {
  __shared__ double t[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = bx + threadIdx.x, c = by + k;
    t[k][threadIdx.x] = (r < n && c < n) ? in[idx(r, c, ldi)] : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = by + threadIdx.x, c = bx + k;
    if (r < n && c < n) out[idx(r, c, n)] = t[threadIdx.x][k];
  }
}

// Diagonal-block inverses of the transposed factor: block i of `inv` holds
// inv(L_ii) then inv(U_ii) (64 x 64 each, column-major); block i of `out`
// gets inv(U_ii)^T = inv(U_ii^T) (the lower slot: U^T is the lower factor of
// the transpose) then inv(L_ii)^T (the upper slot).
__global__ void transpose_inverses_kernel(const double* __restrict__ inv, double* out, int blocks) {
  constexpr int B = 64;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 2LL * B * B * blocks;
       e += (long long)gridDim.x * blockDim.x) {
    const long long blk = e / (2 * B * B);
    const int w = (int)(e % (2 * B * B));
    const int slot = w / (B * B), el = w % (B * B), r = el % B, c = el / B;
    const double* src = inv + blk * 2 * B * B + (slot == 0 ? B * B : 0);
    out[e] = src[r * B + c];
  }
}

// out[c] = sum_i |A(i, c)| over the n x n matrix, one warp per column; out
// is the column sums (||A||_1 is their maximum).
__global__ void col_abs_sum_kernel(const double* __restrict__ A, long long lda, int n, double* out) {
  const int lane = threadIdx.x & 31;
  const long long c = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (c >= n) return;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += fabs(A[idx(i, c, lda)]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (lane == 0) out[c] = s;
}

int grid_of(long long work) {
  long long g = (work + 255) / 256;
  return (int)std::max(1LL, std::min(g, 148LL * 16));
}

}  // namespace

// T (n x nrhs at leading dimension n) <- U^{-1} L^{-1} T with the compact L\U
// at lu: the two triangular solves in launches of up to tri_solve_rhs_max()
// right-hand sides, each with a fresh epoch of `flags`.
int lu_solve_inplace(const double* lu, long long ldlu, int n, const double* inv, double* T,
                     int nrhs, unsigned* flags, unsigned& epoch, cudaStream_t st) {
  int* status = reinterpret_cast<int*>(flags + tri_solve_flag_count(n));
  const int cmax = tri_solve_rhs_max();
  for (int c0 = 0; c0 < nrhs; c0 += cmax) {
    const int nc = std::min(cmax, nrhs - c0);
    for (int up = 0; up < 2; ++up) {
      if (++epoch == 0) ++epoch;
      const int s = up ? launch_tri_upper(lu, ldlu, n, inv, T + (size_t)c0 * n, n, nc, flags,
                                          epoch, status, st)
                       : launch_tri_lower_unit(lu, ldlu, n, inv, T + (size_t)c0 * n, n, nc,
                                               flags, epoch, status, st);
      if (s != kOk) return s;
    }
  }
  return kOk;
}

// Flags + status word for lu_solve_inplace at order n (zeroed).
int alloc_flags(int n, unsigned** flags, cudaStream_t st) {
  const size_t bytes = sizeof(unsigned) * ((size_t)tri_solve_flag_count(n) + 1);
  if (cudaMallocAsync(reinterpret_cast<void**>(flags), bytes, st) != cudaSuccess) {
    cudaGetLastError();
    *flags = nullptr;
    return kAllocationFailed;
  }
  if (cudaMemsetAsync(*flags, 0, bytes, st) != cudaSuccess) return kCudaFailure;
  return kOk;
}

// kOk, or the status a triangular solve left in the flags' status word
// (synchronises st).
int solve_status(const unsigned* flags, int n, cudaStream_t st) {
  int h = 0;
  if (cudaMemcpyAsync(&h, flags + tri_solve_flag_count(n), sizeof(int), cudaMemcpyDeviceToHost,
                      st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return kCudaFailure;
  return h == 0 ? kOk : h;
}

int getrs_device(int n, int nrhs, const double* lu, int ldlu, const int* ipiv, const int* jpiv,
                 double* B, int ldb, cudaStream_t st) {
  if (n < 0 || nrhs < 0 || ldlu < std::max(1, n) || ldb < std::max(1, n)) return kInvalidArgument;
  if (n == 0 || nrhs == 0) return kOk;
  if (!lu || !B || !ipiv || !jpiv) return kInvalidArgument;
  std::vector<int> row(n), col(n);
  for (int i = 0; i < n; ++i) row[i] = col[i] = i;
  for (int k = 0; k < n; ++k) {
    if (ipiv[k] < k || ipiv[k] >= n || jpiv[k] < k || jpiv[k] >= n) return kInvalidArgument;
    std::swap(row[k], row[ipiv[k]]);
    std::swap(col[k], col[jpiv[k]]);
  }
  int* d_perm = nullptr;
  double* tmp = nullptr;
  unsigned* flags = nullptr;
  unsigned epoch = 0;
  double* inv = nullptr;
  if (alloc_flags(n, &flags, st) != kOk) return kAllocationFailed;
  if (cudaMallocAsync(reinterpret_cast<void**>(&inv), sizeof(double) * tri_inverse_doubles(n),
                      st) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(flags, st);
    return kAllocationFailed;
  }
  if (cudaMallocAsync(reinterpret_cast<void**>(&d_perm), sizeof(int) * 2 * (size_t)n, st) !=
      cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(flags, st);
    cudaFreeAsync(inv, st);
    return kAllocationFailed;
  }
  if (cudaMallocAsync(reinterpret_cast<void**>(&tmp), sizeof(double) * (size_t)n * nrhs, st) !=
      cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(d_perm, st);
    cudaFreeAsync(flags, st);
    cudaFreeAsync(inv, st);
    return kAllocationFailed;
  }
  int status = kOk;
  if (cudaMemcpyAsync(d_perm, row.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemcpyAsync(d_perm + n, col.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st) !=
          cudaSuccess)
    status = kCudaFailure;
  if (status == kOk) {
    const long long total = (long long)n * nrhs;
    dp::note_launch();
    gather_rows_kernel<<<grid_of(total), 256, 0, st>>>(B, ldb, tmp, n, d_perm, n, nrhs);
    status = launch_diag_inverse(lu, ldlu, n, inv, st);
    if (status == kOk) status = lu_solve_inplace(lu, ldlu, n, inv, tmp, nrhs, flags, epoch, st);
    if (status == kOk) {
      dp::note_launch();
      scatter_rows_kernel<<<grid_of(total), 256, 0, st>>>(tmp, n, B, ldb, d_perm + n, n, nrhs);
    }
    if (cudaGetLastError() != cudaSuccess && status == kOk) status = kCudaFailure;
    if (status == kOk) status = solve_status(flags, n, st);
  }
  cudaFreeAsync(tmp, st);
  cudaFreeAsync(d_perm, st);
  cudaFreeAsync(flags, st);
  cudaFreeAsync(inv, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && status == kOk) status = kCudaFailure;
  return status;
}

namespace {

// max over columns of ||R_c|| / (normA ||X_c|| + ||B_c||), all infinity norms.
int backward_error(const double* A, int lda, int n, const double* B, int ldb, const double* X,
                   int ldx, int nrhs, double* R, double* norms, double normA,
                   const std::vector<double>& normB, double& berr, cudaStream_t st) {
  const long long total = (long long)n * nrhs;
  dp::note_launch();
  copy_kernel<<<grid_of(total), 256, 0, st>>>(B, ldb, R, n, n, nrhs);
  launch_gemm_minus(n, nrhs, n, A, lda, X, ldx, R, n, st);
  if (cudaMemsetAsync(norms, 0, sizeof(double) * 2 * nrhs, st) != cudaSuccess) return kCudaFailure;
  dim3 g((unsigned)std::min(64, (n + 255) / 256), (unsigned)nrhs);
  dp::note_launch();
  colmax_kernel<<<g, 256, 0, st>>>(R, n, n, nrhs, norms);
  dp::note_launch();
  colmax_kernel<<<g, 256, 0, st>>>(X, ldx, n, nrhs, norms + nrhs);
  std::vector<double> h(2 * (size_t)nrhs);
  if (cudaMemcpyAsync(h.data(), norms, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return kCudaFailure;
  berr = 0.0;
  for (int c = 0; c < nrhs; ++c) {
    const double den = normA * h[nrhs + c] + normB[c];
    const double e = den > 0.0 ? h[c] / den : (h[c] > 0.0 ? INFINITY : 0.0);
    berr = std::max(berr, std::isnan(e) ? INFINITY : e);
  }
  return kOk;
}

}  // namespace

namespace {

// lu <- A, factor at `prec`, composite orders to the device.
int factorize(Factor& f, const double* A, int lda, int prec, cudaStream_t st) {
  const int n = f.n;
  dp::note_launch();
  copy_kernel<<<grid_of((long long)n * n), 256, 0, st>>>(A, lda, f.lu, n, n, n);
  dp_options opt;
  dp_options_init(&opt);
  opt.precision = prec;
  opt.panel_rows = f.panel_rows;
  int info = -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  const int s = getrf_device(n, n, f.lu, n, f.ipiv.data(), f.jpiv.data(), &info, st, &opt);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  f.factor_ms += ms;
  f.info = info;
  f.precision = prec;
  if (s != kOk || info < n) return s;
  std::vector<int> order(2 * (size_t)n);
  for (int i = 0; i < n; ++i) order[i] = order[n + i] = i;
  for (int k = 0; k < n; ++k) {
    std::swap(order[k], order[f.ipiv[k]]);
    std::swap(order[n + k], order[n + f.jpiv[k]]);
  }
  if (cudaMemcpyAsync(f.d_perm, order.data(), sizeof(int) * 2 * (size_t)n, cudaMemcpyHostToDevice,
                      st) != cudaSuccess ||
      launch_diag_inverse(f.lu, n, n, f.d_inv, st) != kOk || cudaStreamSynchronize(st) != cudaSuccess)
    return kCudaFailure;
  return kOk;
}

// X = A^{-1} B through the factors (X, tmp: n x nrhs, leading dimension n).
int solve_with(Factor& f, const double* B, int ldb, double* X, double* tmp, int nrhs,
               cudaStream_t st) {
  const int n = f.n;
  const long long total = (long long)n * nrhs;
  dp::note_launch();
  gather_rows_kernel<<<grid_of(total), 256, 0, st>>>(B, ldb, tmp, n, f.d_perm, n, nrhs);
  const int s = lu_solve_inplace(f.lu, n, n, f.d_inv, tmp, nrhs, f.d_flags, f.epoch, st);
  if (s != kOk) return s;
  dp::note_launch();
  scatter_rows_kernel<<<grid_of(total), 256, 0, st>>>(tmp, n, X, n, f.d_perm + n, n, nrhs);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

// z = A^{-T} c through the factors: A^T = Q U^T L^T P, so with w[k] =
// c[col[k]]: U^T v = w (lower solve on the transposed factor T = (L\U)^T),
// L^T u = v (upper solve on T), z[row[k]] = u[k].  `lut` / `inv_t` are the
// transpose of the compact factor and its transposed diagonal inverses.
int solve_transposed(Factor& f, const double* lut, const double* inv_t, const double* c, double* z,
                     double* tmp, cudaStream_t st) {
  const int n = f.n;
  dp::note_launch();
  gather_rows_kernel<<<grid_of(n), 256, 0, st>>>(c, n, tmp, n, f.d_perm + n, n, 1);
  int* status = reinterpret_cast<int*>(f.d_flags + tri_solve_flag_count(n));
  for (int up = 0; up < 2; ++up) {
    if (++f.epoch == 0) ++f.epoch;
    const int s = up ? launch_tri_upper(lut, n, n, inv_t, tmp, n, 1, f.d_flags, f.epoch, status, st)
                     : launch_tri_lower_unit(lut, n, n, inv_t, tmp, n, 1, f.d_flags, f.epoch,
                                             status, st);
    if (s != kOk) return s;
  }
  dp::note_launch();
  scatter_rows_kernel<<<grid_of(n), 256, 0, st>>>(tmp, n, z, n, f.d_perm, n, 1);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

}  // namespace

// Hager-Higham estimate of ||A^{-1}||_1 from the factors (Hager 1984, with
// Higham's 1988 safeguards as in LAPACK's dlacon: at most 5 iterations, stop
// when the sign vector repeats or the gradient test fails, then take the
// larger of that estimate and 2 ||A^{-1} x||_1 / (3 n) for the alternating
// vector x_i = (-1)^i (1 + i / (n - 1))); kappa_1 = ||A||_1 * estimate.  The
// solves go through the factors held now (mixed factors estimate the
// condition of the matrix they factor exactly, A + E).
int factor_condest(Factor* f, const double* A, int lda, double* kappa, double* inv_norm,
                   cudaStream_t st) {
  if (!f || !kappa || !A || lda < f->n) return kInvalidArgument;
  const int n = f->n;
  *kappa = INFINITY;
  if (inv_norm) *inv_norm = INFINITY;
  if (f->info < n) return kOk;  // singular: infinite condition
  double *lut = nullptr, *inv_t = nullptr, *vec = nullptr;
  auto release = [&] {
    if (lut) cudaFreeAsync(lut, st);
    if (inv_t) cudaFreeAsync(inv_t, st);
    if (vec) cudaFreeAsync(vec, st);
    cudaStreamSynchronize(st);
  };
  const size_t nb = (size_t)(n + 63) / 64;
  if (cudaMallocAsync(reinterpret_cast<void**>(&lut), sizeof(double) * (size_t)n * n, st) !=
          cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&inv_t), sizeof(double) * tri_inverse_doubles(n),
                      st) != cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&vec), sizeof(double) * 4 * (size_t)n, st) !=
          cudaSuccess) {
    cudaGetLastError();
    release();
    return kAllocationFailed;
  }
  double* x = vec;          // input of a solve
  double* y = vec + n;      // its result
  double* tmp = vec + 2 * (size_t)n;
  double* colsum = vec + 3 * (size_t)n;
  dp::note_launch(3);
  transpose_kernel<<<dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, st>>>(f->lu, n, lut, n);
  transpose_inverses_kernel<<<grid_of((long long)(2 * 64 * 64 * nb)), 256, 0, st>>>(f->d_inv, inv_t,
                                                                                  (int)nb);
  col_abs_sum_kernel<<<(int)(((long long)n * 32 + 255) / 256), 256, 0, st>>>(A, lda, n, colsum);
  int status = cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
  std::vector<double> hx(n), hy(n), hsum(n);
  auto down = [&](std::vector<double>& h, const double* d) {
    if (status == kOk && (cudaMemcpyAsync(h.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                          st) != cudaSuccess ||
                          cudaStreamSynchronize(st) != cudaSuccess))
      status = kCudaFailure;
  };
  auto up = [&](const std::vector<double>& h, double* d) {
    if (status == kOk &&
        cudaMemcpyAsync(d, h.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st) != cudaSuccess)
      status = kCudaFailure;
  };
  auto forward = [&] {  // y = A^{-1} x (x on the device), copied to hy
    if (status == kOk) status = solve_with(*f, x, n, y, tmp, 1, st);
    down(hy, y);
  };
  auto backward = [&] {  // y = A^{-T} x, copied to hy
    if (status == kOk) status = solve_transposed(*f, lut, inv_t, x, y, tmp, st);
    down(hy, y);
  };
  down(hsum, colsum);
  double normA = 0.0;
  for (double v : hsum) normA = std::max(normA, std::isnan(v) ? INFINITY : v);
  double est = 0.0;
  if (n == 1) {
    hx[0] = 1.0;
    up(hx, x);
    forward();
    est = std::fabs(hy[0]);
  } else {
    std::vector<double> sign(n, 0.0);
    for (int i = 0; i < n; ++i) hx[i] = 1.0 / n;
    up(hx, x);
    forward();
    int jlast = -1;
    for (int it = 0; it < 5 && status == kOk; ++it) {
      double s1 = 0.0;
      for (double v : hy) s1 += std::fabs(v);
      if (it > 0 && s1 <= est) break;  // no increase
      est = s1;
      bool same = it > 0;
      for (int i = 0; i < n; ++i) {
        const double sg = hy[i] >= 0.0 ? 1.0 : -1.0;
        same = same && sg == sign[i];
        sign[i] = sg;
      }
      if (same) break;  // the sign vector repeats: converged
      up(sign, x);
      backward();       // z = A^{-T} sign
      int j = 0;
      for (int i = 1; i < n; ++i)
        if (std::fabs(hy[i]) > std::fabs(hy[j])) j = i;
      if (it > 0 && j == jlast) break;
      double zx = 0.0;
      for (int i = 0; i < n; ++i) zx += hy[i] * hx[i];
      if (it > 0 && std::fabs(hy[j]) <= zx) break;  // gradient test
      jlast = j;
      std::fill(hx.begin(), hx.end(), 0.0);
      hx[j] = 1.0;
      up(hx, x);
      forward();
    }
    // alternating-sign vector safeguard
    for (int i = 0; i < n; ++i)
      hx[i] = ((i & 1) ? -1.0 : 1.0) * (1.0 + (double)i / (double)(n - 1));
    up(hx, x);
    forward();
    double s1 = 0.0;
    for (double v : hy) s1 += std::fabs(v);
    est = std::max(est, 2.0 * s1 / (3.0 * n));
  }
  if (status == kOk && f->d_flags) status = solve_status(f->d_flags, n, st);
  release();
  if (status != kOk) return status;
  if (inv_norm) *inv_norm = est;
  *kappa = normA * est;
  return kOk;
}

void factor_destroy(Factor* f, cudaStream_t st) {
  if (!f) return;
  if (f->lu) cudaFreeAsync(f->lu, st);
  if (f->d_perm) cudaFreeAsync(f->d_perm, st);
  if (f->d_flags) cudaFreeAsync(f->d_flags, st);
  if (f->d_inv) cudaFreeAsync(f->d_inv, st);
  cudaStreamSynchronize(st);
  delete f;
}

size_t factor_bytes(int n) {
  return sizeof(double) * ((size_t)n * n + tri_inverse_doubles(n)) + sizeof(int) * 2 * (size_t)n +
         sizeof(unsigned) * ((size_t)tri_solve_flag_count(n) + 1);
}

int factor_create(Factor** out, int n, const double* A, int lda, int precision, cudaStream_t st,
                  int panel_rows) {
  if (!out) return kInvalidArgument;
  *out = nullptr;
  if (n < 1 || lda < n || !A ||
      !valid_precision(precision))
    return kInvalidArgument;
  auto* f = new (std::nothrow) Factor;
  if (!f) return kAllocationFailed;
  f->n = n;
  f->panel_rows = std::max(0, panel_rows);
  f->ipiv.resize(n);
  f->jpiv.resize(n);
  double* normA = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&f->lu), sizeof(double) * (size_t)n * n, st) !=
          cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&f->d_perm), sizeof(int) * 2 * (size_t)n, st) !=
          cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&normA), sizeof(double), st) != cudaSuccess) {
    cudaGetLastError();
    if (normA) cudaFreeAsync(normA, st);
    factor_destroy(f, st);
    return kAllocationFailed;
  }
  int status = alloc_flags(n, &f->d_flags, st);
  if (status == kOk &&
      cudaMallocAsync(reinterpret_cast<void**>(&f->d_inv), sizeof(double) * tri_inverse_doubles(n),
                      st) != cudaSuccess) {
    cudaGetLastError();
    f->d_inv = nullptr;
    status = kAllocationFailed;
  }
  if (status != kOk) {
    cudaFreeAsync(normA, st);
    factor_destroy(f, st);
    return status;
  }
  if (cudaMemsetAsync(normA, 0, sizeof(double), st) != cudaSuccess) status = kCudaFailure;
  if (status == kOk) {
    dp::note_launch();
    row_abs_sum_kernel<<<(n + 255) / 256, 256, 0, st>>>(A, lda, n, normA);
    if (cudaMemcpyAsync(&f->normA, normA, sizeof(double), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      status = kCudaFailure;
  }
  if (status == kOk) status = factorize(*f, A, lda, precision, st);
  if (status == kOk && f->precision != DP_PRECISION_FP64 && f->info == n) {
    // Screen of the mixed-precision factors: max |u_ii| / min |u_ii| bounds
    // kappa(U) from below, and refinement contracts only while kappa times
    // the factors' error (about 2^-24 for BF16x6) stays well below one; a
    // ratio beyond kMixedPivotRatio means refinement would stall, so the
    // factors are replaced by plain FP64 ones before any solve.
    double range[2] = {0.0, INFINITY};
    double* scr = nullptr;
    if (status == kOk &&
        cudaMallocAsync(reinterpret_cast<void**>(&scr), 2 * sizeof(double), st) != cudaSuccess) {
      cudaGetLastError();
      status = kAllocationFailed;
    }
    if (status == kOk) {
      if (cudaMemcpyAsync(scr, range, sizeof(range), cudaMemcpyHostToDevice, st) != cudaSuccess)
        status = kCudaFailure;
      dp::note_launch();
      diag_range_kernel<<<std::min(64, (n + 255) / 256), 256, 0, st>>>(f->lu, n, n, scr);
      if (status == kOk &&
          (cudaMemcpyAsync(range, scr, sizeof(range), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
           cudaStreamSynchronize(st) != cudaSuccess))
        status = kCudaFailure;
      cudaFreeAsync(scr, st);
    }
    if (status == kOk && !(range[0] <= kMixedPivotRatio * range[1])) {
      f->refactored = 1;
      status = factorize(*f, A, lda, DP_PRECISION_FP64, st);
    }
  }
  cudaFreeAsync(normA, st);
  if (status != kOk) {
    factor_destroy(f, st);
    return status;
  }
  *out = f;
  return kOk;
}

// Solve A X = B with the factors and FP64 refinement (A: the matrix the
// factors came from, B overwritten with X).  A refinement on mixed-precision
// factors that stalls (error not halved) or misses the tolerance re-factors
// A in plain FP64 - the factors stay FP64 for later solves.
int factor_solve(Factor* f, const double* A, int lda, double* B, int ldb, int nrhs, int max_iter,
                 double tol, dp_ir_result* res, cudaStream_t st) {
  if (!res) return kInvalidArgument;
  std::memset(res, 0, sizeof(*res));
  res->info = f ? f->info : -1;
  res->backward_error = INFINITY;
  if (!f || nrhs < 0 || lda < f->n || ldb < f->n || max_iter < 0 || !(tol >= 0.0) || !A ||
      (nrhs > 0 && !B))
    return kInvalidArgument;
  const int n = f->n;
  if (f->info < n && f->precision != DP_PRECISION_FP64) {
    // a mixed-precision factorisation that delayed: decide in plain FP64
    f->refactored = 1;
    const double fms0 = f->factor_ms;
    const int s = factorize(*f, A, lda, DP_PRECISION_FP64, st);
    res->factor_ms = f->factor_ms - fms0;
    res->info = f->info;
    res->refactored = 1;
    if (s != kOk) return s;
  }
  if (f->info < n) return kOk;  // singular: no solution
  if (nrhs == 0) {
    res->backward_error = 0.0;
    res->converged = 1;
    return kOk;
  }
  const size_t nr = (size_t)n * nrhs;
  double *X = nullptr, *R = nullptr, *T = nullptr, *norms = nullptr;
  auto release = [&] {
    if (X) cudaFreeAsync(X, st);
    if (R) cudaFreeAsync(R, st);
    if (T) cudaFreeAsync(T, st);
    if (norms) cudaFreeAsync(norms, st);
    cudaStreamSynchronize(st);
  };
  if (cudaMallocAsync(reinterpret_cast<void**>(&X), nr * sizeof(double), st) != cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&R), nr * sizeof(double), st) != cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&T), nr * sizeof(double), st) != cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&norms), 2 * (size_t)nrhs * sizeof(double), st) !=
          cudaSuccess) {
    cudaGetLastError();
    release();
    return kAllocationFailed;
  }
  std::vector<double> normB(nrhs);
  int status = kOk;
  {
    if (cudaMemsetAsync(norms, 0, sizeof(double) * nrhs, st) != cudaSuccess) status = kCudaFailure;
    dim3 g((unsigned)std::min(64, (n + 255) / 256), (unsigned)nrhs);
    dp::note_launch();
    colmax_kernel<<<g, 256, 0, st>>>(B, ldb, n, nrhs, norms);
    if (status == kOk &&
        (cudaMemcpyAsync(normB.data(), norms, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st) !=
             cudaSuccess ||
         cudaStreamSynchronize(st) != cudaSuccess))
      status = kCudaFailure;
  }

  auto refine = [&](int iters_left, bool& converged) -> int {
    converged = false;
    double prev = INFINITY;
    for (int it = 0;; ++it) {
      double berr = INFINITY;
      int s = backward_error(A, lda, n, B, ldb, X, n, nrhs, R, norms, f->normA, normB, berr, st);
      if (s != kOk) return s;
      res->backward_error = berr;
      if (berr <= tol) {
        converged = true;
        return kOk;
      }
      if (it >= iters_left) return kOk;
      if (it > 0 && !(berr <= 0.5 * prev)) return kOk;  // stalled
      // converging, but too slowly to reach tol within the steps left: the
      // contraction rate of refinement is about constant (kappa times the
      // factors' error), so stop now rather than after the last step
      if (it > 0 && berr > 0.0 && tol > 0.0) {
        const double needed = std::log(tol / berr) / std::log(berr / prev);
        if (it + needed > iters_left + 0.5) return kOk;
      }
      prev = berr;
      s = solve_with(*f, R, n, R, T, nrhs, st);
      if (s != kOk) return s;
      dp::note_launch();
      axpy_kernel<<<grid_of((long long)nr), 256, 0, st>>>(R, n, X, n, n, nrhs);
      res->iterations += 1;
    }
  };

  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, st);
  const double fms0 = f->factor_ms - res->factor_ms;
  bool converged = false;
  if (status == kOk) {
    status = solve_with(*f, B, ldb, X, T, nrhs, st);
    if (status == kOk) status = refine(max_iter, converged);
  }
  if (status == kOk && !converged && f->precision != DP_PRECISION_FP64) {
    // the mixed-precision factors cannot carry this matrix: plain FP64
    f->refactored = 1;
    status = factorize(*f, A, lda, DP_PRECISION_FP64, st);
    if (status == kOk && f->info == n) {
      status = solve_with(*f, B, ldb, X, T, nrhs, st);
      if (status == kOk) status = refine(max_iter, converged);
    }
  }
  cudaEventRecord(t1, st);
  cudaEventSynchronize(t1);
  float tot = 0.f;
  cudaEventElapsedTime(&tot, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (status == kOk) status = solve_status(f->d_flags, n, st);
  res->total_ms = tot;
  res->factor_ms = f->factor_ms - fms0;
  res->info = f->info;
  res->refactored = f->refactored;
  res->converged = converged ? 1 : 0;
  if (status == kOk && f->info == n) {
    dp::note_launch();
    copy_kernel<<<grid_of((long long)nr), 256, 0, st>>>(X, n, B, ldb, n, nrhs);
  }
  release();
  return status;
}

int gesv_ir_device(int n, int nrhs, const double* A, int lda, double* B, int ldb, int precision,
                   int max_iter, double tol, dp_ir_result* res, cudaStream_t st) {
  if (!res) return kInvalidArgument;
  std::memset(res, 0, sizeof(*res));
  res->info = -1;
  res->backward_error = INFINITY;
  if (n < 0 || nrhs < 0 || lda < std::max(1, n) || ldb < std::max(1, n) || max_iter < 0 ||
      !(tol >= 0.0) || !valid_precision(precision))
    return kInvalidArgument;
  if (n == 0 || nrhs == 0) {
    res->info = n;
    res->backward_error = 0.0;
    res->converged = 1;
    return kOk;
  }
  if (!A || !B) return kInvalidArgument;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, st);
  Factor* f = nullptr;
  int status = factor_create(&f, n, A, lda, precision, st);
  const double factor_ms = f ? f->factor_ms : 0.0;
  if (status == kOk) {
    status = factor_solve(f, A, lda, B, ldb, nrhs, max_iter, tol, res, st);
    res->factor_ms += factor_ms;
  }
  if (f) factor_destroy(f, st);
  cudaEventRecord(t1, st);
  cudaEventSynchronize(t1);
  float tot = 0.f;
  cudaEventElapsedTime(&tot, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  res->total_ms = tot;
  return status;
}

}  // namespace dp

extern "C" {

int dp_getrs_device(int n, int nrhs, const double* d_lu, int ldlu, const int* ipiv,
                    const int* jpiv, double* d_b, int ldb, void* stream) {
  return dp::getrs_device(n, nrhs, d_lu, ldlu, ipiv, jpiv, d_b, ldb,
                          static_cast<cudaStream_t>(stream));
}

int dp_gesv_ir_device(int n, int nrhs, const double* d_a, int lda, double* d_b, int ldb,
                      int precision, int max_iter, double tol, dp_ir_result* result, void* stream) {
  return dp::gesv_ir_device(n, nrhs, d_a, lda, d_b, ldb, precision, max_iter, tol, result,
                            static_cast<cudaStream_t>(stream));
}

struct dp_factor {
  dp::Factor* f;
};

int dp_factor_create(dp_factor** out, int n, const double* d_a, int lda, int precision,
                     void* stream) {
  if (!out) return DP_INVALID_ARGUMENT;
  *out = nullptr;
  dp::Factor* f = nullptr;
  const int s = dp::factor_create(&f, n, d_a, lda, precision, static_cast<cudaStream_t>(stream));
  if (s != DP_SUCCESS) return s;
  *out = new (std::nothrow) dp_factor{f};
  if (!*out) {
    dp::factor_destroy(f, static_cast<cudaStream_t>(stream));
    return DP_ALLOCATION_FAILED;
  }
  return DP_SUCCESS;
}

int dp_factor_info(const dp_factor* h, int* info, int* precision, double* factor_ms) {
  if (!h) return DP_INVALID_ARGUMENT;
  if (info) *info = h->f->info;
  if (precision) *precision = h->f->precision;
  if (factor_ms) *factor_ms = h->f->factor_ms;
  return DP_SUCCESS;
}

int dp_factor_solve(dp_factor* h, const double* d_a, int lda, double* d_b, int ldb, int nrhs,
                    int max_iter, double tol, dp_ir_result* result, void* stream) {
  if (!h) return DP_INVALID_ARGUMENT;
  return dp::factor_solve(h->f, d_a, lda, d_b, ldb, nrhs, max_iter, tol, result,
                          static_cast<cudaStream_t>(stream));
}

int dp_factor_condest(dp_factor* h, const double* d_a, int lda, double* kappa1, void* stream) {
  if (!h) return DP_INVALID_ARGUMENT;
  return dp::factor_condest(h->f, d_a, lda, kappa1, nullptr, static_cast<cudaStream_t>(stream));
}

void dp_factor_destroy(dp_factor* h, void* stream) {
  if (!h) return;
  dp::factor_destroy(h->f, static_cast<cudaStream_t>(stream));
  delete h;
}

}  // extern "C"
