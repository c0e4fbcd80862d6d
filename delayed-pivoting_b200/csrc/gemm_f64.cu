// FP64 Schur-complement update  C -= A * B  on the DMMA tensor-core path.
//
// This is the O(n^3) work of the LU: finish_panel's dgemm
// (delayed_lu/delayed_dgetrf.cpp:80-83, delayed_lu_cuda/delayed_dgetrf_cuda.cu:205-209)
// and the far-column update of materialize_partial_panel (:120-123).  The
// inner dimension K is the panel width (<= 256).
//
// sm_100a has no FP64 kind of tcgen05.mma; the FP64 tensor path is
// mma.sync.m16n8k4.f64 (measured at ~37 TFLOP/s on B200, the same rate as
// DFMA).  CTA tile 128 x 128, 8 warps as 2 x 4, warp tile 64 x 32 (4 x 4
// MMAs per k-step), K streamed in chunks of 32 through a 3-stage cp.async
// pipeline into padded shared tiles (A k-major with stride 136, B n-major
// with stride 36: both give conflict-free fragment loads).  The C tile is
// prefetched into L2 when the CTA starts, so the read-modify-write in the
// epilogue does not wait on HBM.  Accumulation is C - sum_k(a*b) with the
// sum formed in FP64 by the tensor core.
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3;
constexpr int LDA_S = BM + 8;  // doubles; == 8 (mod 16)
constexpr int LDB_S = BK + 4;  // doubles; == 4 (mod 16)
constexpr int kGemmThreads = 256;
constexpr int A_STAGE = BK * LDA_S;  // doubles
constexpr int B_STAGE = BN * LDB_S;
constexpr size_t kGemmSmem = (size_t)STAGES * (A_STAGE + B_STAGE) * sizeof(double);

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem), "r"(sz)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mma_f64_16x8x4(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__global__ void __launch_bounds__(kGemmThreads, 1)
dgemm_minus_kernel(int M, int N, int K, const double* __restrict__ A, long long lda,
                   const double* __restrict__ B, long long ldb, double* C, long long ldc) {
  extern __shared__ __align__(16) double gsm[];
  double* As = gsm;                      // [STAGES][BK][LDA_S]
  double* Bs = gsm + STAGES * A_STAGE;   // [STAGES][BN][LDB_S]

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps
  const int g = lane >> 2, t = lane & 3;
  const long long m0 = (long long)blockIdx.x * BM;
  const long long n0 = (long long)blockIdx.y * BN;

  // Prefetch this CTA's C tile into L2 (128-byte lines, in-bounds only).
  {
    const int rows = (int)min((long long)BM, M - m0);
    const int cols = (int)min((long long)BN, N - n0);
    const int lines_per_col = (rows * 8 + 127) / 128 + 1;
    for (int e = tid; e < cols * lines_per_col; e += kGemmThreads) {
      const int c = e / lines_per_col, l = e % lines_per_col;
      const int r = min(rows - 1, l * 16);
      const double* p = C + idx(m0 + r, n0 + c, ldc);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  }

  const int ktiles = (K + BK - 1) / BK;

  auto load_stage = [&](int stage, int kt) {
    double* as = As + stage * A_STAGE;
    double* bs = Bs + stage * B_STAGE;
    const int k0 = kt * BK;
#pragma unroll
    for (int i = 0; i < (BM * BK) / kGemmThreads; ++i) {
      const int e = tid + i * kGemmThreads;
      const int r = e % BM, kk = e / BM;
      const bool ok = (m0 + r < M) && (k0 + kk < K);
      const double* src = ok ? A + idx(m0 + r, k0 + kk, lda) : A;
      cp_async8(as + kk * LDA_S + r, src, ok);
    }
#pragma unroll
    for (int i = 0; i < (BN * BK) / kGemmThreads; ++i) {
      const int e = tid + i * kGemmThreads;
      const int kk = e % BK, c = e / BK;
      const bool ok = (n0 + c < N) && (k0 + kk < K);
      const double* src = ok ? B + idx(k0 + kk, n0 + c, ldb) : B;
      cp_async8(bs + c * LDB_S + kk, src, ok);
    }
  };

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < ktiles) load_stage(nk % STAGES, nk);
      cp_async_commit();
    }
    const double* as = As + (kt % STAGES) * A_STAGE;
    const double* bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[4][2], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        const double* ap = as + (kk + t) * LDA_S + wm * 64 + mi * 16 + g;
        af[mi][0] = ap[0];
        af[mi][1] = ap[8];
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = bs[(wn * 32 + ni * 8 + g) * LDB_S + kk + t];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) mma_f64_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
    }
  }
  cp_async_wait<0>();

  // Epilogue: C -= acc.
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const long long r = m0 + wm * 64 + mi * 16 + g + 8 * (v >> 1);
        const long long c = n0 + wn * 32 + ni * 8 + 2 * t + (v & 1);
        if (r < M && c < N) {
          double* cp = C + idx(r, c, ldc);
          *cp = *cp - acc[mi][ni][v];
        }
      }
    }
  }
}

}  // namespace

void launch_gemm_minus(int M, int N, int K, const double* A, long long lda, const double* B,
                       long long ldb, double* C, long long ldc, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return;
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(dgemm_minus_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kGemmSmem);
    configured = true;
  }
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
  dgemm_minus_kernel<<<grid, kGemmThreads, kGemmSmem, s>>>(M, N, K, A, lda, B, ldb, C, ldc);
}

}  // namespace dp
