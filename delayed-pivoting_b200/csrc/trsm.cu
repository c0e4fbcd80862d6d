// Unit-lower triangular solve of the panel's block row:
//   U12 <- L11^{-1} A12
// (delayed_lu/delayed_dgetrf.cpp:72-74 `cblas_dtrsm(Left, Lower, NoTrans,
// Unit)`; also the first half of materialize_partial_panel, :111-114).
//
// One CTA per 64-column tile of A12.  L11 (w x w, w <= 128) and the tile are
// staged in shared memory; the forward substitution runs column-parallel with
// a CTA barrier per pivot row.  The diagonal of L11 is never read (unit).
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int kTrsmThreads = 256;
constexpr int kTrsmCols = 64;
constexpr int kTrsmMaxW = 128;

__global__ void __launch_bounds__(kTrsmThreads)
trsm_unit_lower_kernel(double* a, long long lda, int r0, int w, int c0, int nc) {
  extern __shared__ __align__(16) double tsm[];
  double* Ls = tsm;                    // [w][w] column-major
  double* Bs = tsm + (size_t)w * w;    // [kTrsmCols][w]
  const int tid = threadIdx.x;
  const int col0 = c0 + blockIdx.x * kTrsmCols;
  const int ncols = min(kTrsmCols, c0 + nc - col0);

  for (int e = tid; e < w * w; e += blockDim.x) {
    const int r = e % w, c = e / w;
    Ls[e] = (r > c) ? a[idx(r0 + r, r0 + c, lda)] : 0.0;
  }
  for (int e = tid; e < w * ncols; e += blockDim.x) {
    const int r = e % w, c = e / w;
    Bs[e] = a[idx(r0 + r, col0 + c, lda)];
  }
  __syncthreads();

  const int c = tid % kTrsmCols;
  const int g = tid / kTrsmCols;            // 4 row groups
  const int groups = blockDim.x / kTrsmCols;
  for (int p = 0; p < w - 1; ++p) {
    if (c < ncols) {
      const double x = Bs[(size_t)c * w + p];
      for (int r = p + 1 + g; r < w; r += groups) Bs[(size_t)c * w + r] -= Ls[(size_t)p * w + r] * x;
    }
    __syncthreads();
  }

  for (int e = tid; e < w * ncols; e += blockDim.x) {
    const int r = e % w, cc = e / w;
    a[idx(r0 + r, col0 + cc, lda)] = Bs[e];
  }
}

}  // namespace

void launch_trsm_unit_lower(double* a, long long lda, int r0, int w, int c0, int nc,
                            cudaStream_t s) {
  if (w <= 1 || nc <= 0) return;  // w == 1: unit diagonal, nothing to solve
  const size_t smem = ((size_t)w * w + (size_t)kTrsmCols * w) * sizeof(double);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(trsm_unit_lower_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(((size_t)kTrsmMaxW * kTrsmMaxW + (size_t)kTrsmCols * kTrsmMaxW) *
                               sizeof(double)));
    configured = true;
  }
  const int grid = (nc + kTrsmCols - 1) / kTrsmCols;
  trsm_unit_lower_kernel<<<grid, kTrsmThreads, smem, s>>>(a, lda, r0, w, c0, nc);
}

}  // namespace dp
