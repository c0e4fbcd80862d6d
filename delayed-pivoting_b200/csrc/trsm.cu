// Unit-lower triangular solve of the panel's block row:
//   U12 <- L11^{-1} A12
// (delayed_lu/delayed_dgetrf.cpp:72-74 `cblas_dtrsm(Left, Lower, NoTrans,
// Unit)`; also the first half of materialize_partial_panel, :111-114).
//
// Diagonal blocks are at most 64 wide (wider blocks are split by the host
// into 64-wide solves and GEMM updates).  A CTA owns 64 columns of A12 and
// two threads own each column, one per 32-row half, with their half in 32
// registers and the forward substitution fully unrolled:
//   phase 1: rows 0..31  <- L(0:32, 0:32)^{-1} rows 0..31
//   phase 2: rows 32..63 <- L(32:64, 32:64)^{-1} (rows 32..63 - L(32:64, 0:32) rows 0..31)
// L11 sits in shared memory (every load of it is a broadcast); the tile is
// staged through shared memory so global loads and stores stay coalesced.
// Rows / columns of L11 beyond w are zero, so narrower blocks run the same
// code.
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int kTrsmW = 64;     // maximum block width
constexpr int kHalf = 32;
constexpr int kTrsmCols = 64;  // columns per CTA
constexpr int kTrsmThreads = 2 * kTrsmCols;
constexpr int kStage = kTrsmW + 1;  // odd stride: conflict-free per-thread column access
constexpr size_t kTrsmSmem = (size_t)(kTrsmW * kTrsmW + kTrsmCols * kStage) * sizeof(double);

__global__ void __launch_bounds__(kTrsmThreads)
trsm_unit_lower_kernel(double* a, long long lda, int r0, int w, int c0, int nc) {
  extern __shared__ __align__(16) double tsm[];
  double* Ls = tsm;                   // Ls[p * 64 + i] = L(i, p), zero outside the strict lower part
  double* Bt = tsm + kTrsmW * kTrsmW;  // Bt[c * 65 + i] = A12(i, c)
  const int tid = threadIdx.x;
  const int col0 = c0 + blockIdx.x * kTrsmCols;
  const int ncols = min(kTrsmCols, c0 + nc - col0);

  for (int e = tid; e < kTrsmW * kTrsmW; e += kTrsmThreads) {
    const int i = e % kTrsmW, pcol = e / kTrsmW;
    Ls[e] = (i > pcol && i < w) ? a[idx(r0 + i, r0 + pcol, lda)] : 0.0;
  }
  for (int e = tid; e < w * ncols; e += kTrsmThreads) {
    const int i = e % w, c = e / w;
    Bt[c * kStage + i] = a[idx(r0 + i, col0 + c, lda)];
  }
  __syncthreads();

  const int c = tid % kTrsmCols;
  const bool upper_half = tid < kTrsmCols;  // warps 0-1: rows 0..31, warps 2-3: rows 32..63
  double* bc = Bt + c * kStage;
  if (upper_half && c < ncols) {
    double x[kHalf];
#pragma unroll
    for (int i = 0; i < kHalf; ++i) x[i] = i < w ? bc[i] : 0.0;
#pragma unroll
    for (int p = 0; p < kHalf - 1; ++p) {
#pragma unroll
      for (int i = p + 1; i < kHalf; ++i) x[i] -= Ls[p * kTrsmW + i] * x[p];
    }
#pragma unroll
    for (int i = 0; i < kHalf; ++i)
      if (i < w) bc[i] = x[i];
  }
  __syncthreads();
  if (!upper_half && c < ncols && w > kHalf) {
    double x[kHalf];
#pragma unroll
    for (int i = 0; i < kHalf; ++i) x[i] = kHalf + i < w ? bc[kHalf + i] : 0.0;
#pragma unroll 4
    for (int p = 0; p < kHalf; ++p) {
      const double xp = bc[p];
#pragma unroll
      for (int i = 0; i < kHalf; ++i) x[i] -= Ls[p * kTrsmW + kHalf + i] * xp;
    }
#pragma unroll
    for (int p = 0; p < kHalf - 1; ++p) {
#pragma unroll
      for (int i = p + 1; i < kHalf; ++i) x[i] -= Ls[(kHalf + p) * kTrsmW + kHalf + i] * x[p];
    }
#pragma unroll
    for (int i = 0; i < kHalf; ++i)
      if (kHalf + i < w) bc[kHalf + i] = x[i];
  }
  __syncthreads();
  for (int e = tid; e < w * ncols; e += kTrsmThreads) {
    const int i = e % w, cc = e / w;
    a[idx(r0 + i, col0 + cc, lda)] = Bt[cc * kStage + i];
  }
}

}  // namespace

int trsm_max_width() { return kTrsmW; }

void launch_trsm_unit_lower(double* a, long long lda, int r0, int w, int c0, int nc,
                            cudaStream_t s) {
  if (w <= 1 || nc <= 0) return;  // w == 1: unit diagonal, nothing to solve
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(trsm_unit_lower_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kTrsmSmem);
    configured = true;
  }
  const int grid = (nc + kTrsmCols - 1) / kTrsmCols;
  trsm_unit_lower_kernel<<<grid, kTrsmThreads, kTrsmSmem, s>>>(a, lda, r0, w, c0, nc);
}

}  // namespace dp
