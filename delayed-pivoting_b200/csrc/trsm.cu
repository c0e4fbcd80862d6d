// Triangular solves with a diagonal block of at most 64 rows:
//   lower, unit diagonal:   B <- L^{-1} B   (the panel's block row, U12 = L11^{-1} A12,
//                           delayed_lu/delayed_dgetrf.cpp:72-74; also the first half of
//                           materialize_partial_panel, :111-114; and the forward
//                           substitution of the solve)
//   upper, non-unit:        B <- U^{-1} B   (back substitution of the solve)
// Wider blocks are split by the host into 64-wide solves and GEMM updates.
//
// A CTA owns 64 columns of B; two threads own each column, one per 32-row
// half, holding their half in 32 registers with the substitution fully
// unrolled.  The triangle sits in shared memory (every load of it is a
// broadcast); the tile is staged through shared memory so the global loads
// and stores stay coalesced.  Rows / columns beyond w are an identity block,
// so narrower blocks run the same code.
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int kTrsmW = 64;     // maximum block width
constexpr int kHalf = 32;
constexpr int kTrsmCols = 64;  // columns per CTA
constexpr int kTrsmThreads = 2 * kTrsmCols;
constexpr int kStage = kTrsmW + 1;  // odd stride: conflict-free per-thread column access
constexpr size_t kTrsmSmem =
    (size_t)(kTrsmW * kTrsmW + kTrsmW + kTrsmCols * kStage) * sizeof(double);

__device__ __forceinline__ void stage_in(const double* B, long long ldb, int w, int ncols,
                                         double* Bt) {
  for (int e = threadIdx.x; e < w * ncols; e += kTrsmThreads) {
    const int i = e % w, c = e / w;
    Bt[c * kStage + i] = B[idx(i, c, ldb)];
  }
}

__device__ __forceinline__ void stage_out(double* B, long long ldb, int w, int ncols,
                                          const double* Bt) {
  for (int e = threadIdx.x; e < w * ncols; e += kTrsmThreads) {
    const int i = e % w, cc = e / w;
    B[idx(i, cc, ldb)] = Bt[cc * kStage + i];
  }
}

// B (w x nc) <- L^{-1} B, L unit lower (w x w).
__global__ void __launch_bounds__(kTrsmThreads)
trsm_lower_unit_kernel(const double* __restrict__ L, long long ldl, double* B, long long ldb, int w,
                       int nc, const int* gate) {
  if (gate && *gate >= 0) return;
  extern __shared__ __align__(16) double tsm[];
  double* Ls = tsm;                    // Ls[p * 64 + i] = L(i, p), zero outside the strict lower part
  double* Bt = tsm + kTrsmW * kTrsmW + kTrsmW;  // Bt[c * 65 + i] = B(i, c)
  const int tid = threadIdx.x;
  const int col0 = blockIdx.x * kTrsmCols;
  const int ncols = min(kTrsmCols, nc - col0);
  B += idx(0, col0, ldb);

  for (int e = tid; e < kTrsmW * kTrsmW; e += kTrsmThreads) {
    const int i = e % kTrsmW, pcol = e / kTrsmW;
    Ls[e] = (i > pcol && i < w) ? L[idx(i, pcol, ldl)] : 0.0;
  }
  stage_in(B, ldb, w, ncols, Bt);
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
  stage_out(B, ldb, w, ncols, Bt);
}

// B (w x nc) <- U^{-1} B, U upper with its diagonal (w x w).
__global__ void __launch_bounds__(kTrsmThreads)
trsm_upper_kernel(const double* __restrict__ U, long long ldu, double* B, long long ldb, int w,
                  int nc) {
  extern __shared__ __align__(16) double tsm[];
  double* Us = tsm;                     // Us[p * 64 + i] = U(i, p) for i < p, zero elsewhere
  double* dg = tsm + kTrsmW * kTrsmW;   // diagonal, 1 beyond w
  double* Bt = dg + kTrsmW;
  const int tid = threadIdx.x;
  const int col0 = blockIdx.x * kTrsmCols;
  const int ncols = min(kTrsmCols, nc - col0);
  B += idx(0, col0, ldb);

  for (int e = tid; e < kTrsmW * kTrsmW; e += kTrsmThreads) {
    const int i = e % kTrsmW, pcol = e / kTrsmW;
    Us[e] = (i < pcol && pcol < w) ? U[idx(i, pcol, ldu)] : 0.0;
  }
  for (int i = tid; i < kTrsmW; i += kTrsmThreads) dg[i] = i < w ? U[idx(i, i, ldu)] : 1.0;
  stage_in(B, ldb, w, ncols, Bt);
  __syncthreads();

  const int c = tid % kTrsmCols;
  const bool top = tid < kTrsmCols;  // warps 0-1: rows 0..31, warps 2-3: rows 32..63
  double* bc = Bt + c * kStage;
  if (!top && c < ncols && w > kHalf) {
    double x[kHalf];
#pragma unroll
    for (int i = 0; i < kHalf; ++i) x[i] = kHalf + i < w ? bc[kHalf + i] : 0.0;
#pragma unroll
    for (int p = kHalf - 1; p >= 0; --p) {
      x[p] /= dg[kHalf + p];
#pragma unroll
      for (int i = 0; i < p; ++i) x[i] -= Us[(kHalf + p) * kTrsmW + kHalf + i] * x[p];
    }
#pragma unroll
    for (int i = 0; i < kHalf; ++i)
      if (kHalf + i < w) bc[kHalf + i] = x[i];
  }
  __syncthreads();
  if (top && c < ncols) {
    double x[kHalf];
#pragma unroll
    for (int i = 0; i < kHalf; ++i) x[i] = i < w ? bc[i] : 0.0;
    if (w > kHalf) {
#pragma unroll 4
      for (int p = 0; p < kHalf; ++p) {
        const double xp = bc[kHalf + p];
#pragma unroll
        for (int i = 0; i < kHalf; ++i) x[i] -= Us[(kHalf + p) * kTrsmW + i] * xp;
      }
    }
#pragma unroll
    for (int p = kHalf - 1; p >= 0; --p) {
      x[p] /= dg[p];
#pragma unroll
      for (int i = 0; i < p; ++i) x[i] -= Us[p * kTrsmW + i] * x[p];
    }
#pragma unroll
    for (int i = 0; i < kHalf; ++i)
      if (i < w) bc[i] = x[i];
  }
  __syncthreads();
  stage_out(B, ldb, w, ncols, Bt);
}

void configure() {
  ensure_smem((const void*)trsm_lower_unit_kernel, kTrsmSmem);
  ensure_smem((const void*)trsm_upper_kernel, kTrsmSmem);
}

}  // namespace

// T <- I - L^{-1} for a unit lower w x w block L (w <= 256), so that the
// block solve X = L^{-1} B becomes the FP64 tensor-core update
// X = B - T B (T strictly lower).  Column j of L^{-1} is one warp's forward
// substitution L x = e_j: lane l holds rows l + 32 r, the entry x_k travels
// by shuffle.  The CTA's 8 warps share L through shared memory: 32-column
// chunks of its strict lower part (zeros elsewhere) are staged by cp.async,
// the next chunk in flight while the warps step through the current one.
constexpr int kInvMaxW = 256;
constexpr int kInvRows = kInvMaxW / 32;  // rows per lane
constexpr int kInvWarps = 8;
constexpr int kInvChunk = 32;            // columns of L per staged chunk
constexpr size_t kInvSmem = 2 * (size_t)kInvChunk * kInvMaxW * sizeof(double);
static_assert(kInvChunk == 32, "one chunk per lane row group");

__device__ __forceinline__ void cp_async8_zfill(double* dst, const double* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(ok ? 8 : 0)
               : "memory");
}

__global__ void __launch_bounds__(32 * kInvWarps)
lower_inverse_kernel(const double* __restrict__ L, long long ldl, int w, double* __restrict__ T,
                     long long ldt) {
  extern __shared__ __align__(16) double ls[];  // [2][kInvChunk][kInvMaxW]
  const int tid = threadIdx.x, lane = tid & 31;
  const int j0 = blockIdx.x * kInvWarps;
  const int j = j0 + (tid >> 5);
  const bool active = j < w;
  double x[kInvRows];
#pragma unroll
  for (int r = 0; r < kInvRows; ++r) x[r] = lane + 32 * r == j ? 1.0 : 0.0;
  const int c_first = j0 / kInvChunk;
  const int c_last = w >= 2 ? (w - 2) / kInvChunk : -1;  // last chunk holding a step
  auto stage = [&](int c, int buf) {
    double* dst = ls + (size_t)buf * kInvChunk * kInvMaxW;
    for (int e = tid; e < kInvChunk * kInvMaxW; e += 32 * kInvWarps) {
      const int kk = e / kInvMaxW, i = e % kInvMaxW;
      const int k = c * kInvChunk + kk;
      const bool ok = i < w && i > k;
      cp_async8_zfill(dst + e, ok ? L + i + (size_t)k * (size_t)ldl : L, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (c_first <= c_last) stage(c_first, 0);
#pragma unroll
  for (int c = 0; c < kInvRows; ++c) {
    if (c < c_first || c > c_last) continue;  // (CTA-uniform)
    const int buf = (c - c_first) & 1;
    if (c + 1 <= c_last) {
      stage(c + 1, buf ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const double* lc = ls + (size_t)buf * kInvChunk * kInvMaxW;
    if (active) {
#pragma unroll
      for (int kk = 0; kk < kInvChunk; ++kk) {
        const int k = kInvChunk * c + kk;
        if (k < j || k >= w - 1) continue;  // (warp-uniform)
        const double xk = __shfl_sync(0xffffffffu, x[c], kk);
#pragma unroll
        for (int r = c; r < kInvRows; ++r)
          x[r] = fma(-lc[kk * kInvMaxW + lane + 32 * r], xk, x[r]);  // zero where i <= k
      }
    }
    __syncthreads();  // this buffer is restaged two chunks later
  }
  if (!active) return;
  double* Tj = T + (size_t)j * (size_t)ldt;
#pragma unroll
  for (int r = 0; r < kInvRows; ++r) {
    const int i = lane + 32 * r;
    if (i < w) Tj[i] = i > j ? -x[r] : 0.0;
  }
}

// dst(0:rows, 0:cols) <- src(0:rows, 0:cols), both column-major: a CTA per
// column at a time, consecutive threads on consecutive rows.
__global__ void __launch_bounds__(256)
copy_block_kernel(const double* __restrict__ src, long long lds, double* __restrict__ dst,
                  long long ldd, int rows, int cols) {
  for (long long c = blockIdx.x; c < cols; c += gridDim.x) {
    const double* s = src + c * lds;
    double* d = dst + c * ldd;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) d[r] = s[r];
  }
}

int trsm_max_width() { return kTrsmW; }

void launch_copy_block(const double* src, long long lds, double* dst, long long ldd, int rows,
                       int cols, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  dp::note_launch();
  copy_block_kernel<<<std::min(cols, 148 * 8), 256, 0, s>>>(src, lds, dst, ldd, rows, cols);
}

int lower_inverse_max_width() { return kInvMaxW; }

void launch_lower_inverse(const double* L, long long ldl, int w, double* T, long long ldt,
                          cudaStream_t s) {
  if (w <= 0) return;
  dp::ensure_smem((const void*)lower_inverse_kernel, kInvSmem);
  dp::note_launch();
  lower_inverse_kernel<<<(w + kInvWarps - 1) / kInvWarps, 32 * kInvWarps, kInvSmem, s>>>(
      L, ldl, w, T, ldt);
}

void launch_trsm_lower_unit(const double* L, long long ldl, double* B, long long ldb, int w, int nc,
                            cudaStream_t s, const int* gate) {
  if (w <= 1 || nc <= 0) return;  // w == 1: unit diagonal, nothing to solve
  configure();
  const int grid = (nc + kTrsmCols - 1) / kTrsmCols;
  dp::note_launch();
  trsm_lower_unit_kernel<<<grid, kTrsmThreads, kTrsmSmem, s>>>(L, ldl, B, ldb, w, nc, gate);
}

void launch_trsm_upper(const double* U, long long ldu, double* B, long long ldb, int w, int nc,
                       cudaStream_t s) {
  if (w <= 0 || nc <= 0) return;
  configure();
  const int grid = (nc + kTrsmCols - 1) / kTrsmCols;
  dp::note_launch();
  trsm_upper_kernel<<<grid, kTrsmThreads, kTrsmSmem, s>>>(U, ldu, B, ldb, w, nc);
}

void launch_trsm_unit_lower(double* a, long long lda, int r0, int w, int c0, int nc,
                            cudaStream_t s, const int* gate) {
  launch_trsm_lower_unit(a + idx(r0, r0, lda), lda, a + idx(r0, c0, lda), lda, w, nc, s, gate);
}

}  // namespace dp
