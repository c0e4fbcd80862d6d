// FP64 Schur-complement update  C -= A * B  on the DMMA tensor-core path.
//
// This is the O(n^3) work of the LU: finish_panel's dgemm
// (delayed_lu/delayed_dgetrf.cpp:80-83, delayed_lu_cuda/delayed_dgetrf_cuda.cu:205-209)
// and the far-column update of materialize_partial_panel (:120-123).  The
// inner dimension K is the (outer) panel width.
//
// sm_100a has no FP64 kind of tcgen05.mma; the FP64 tensor path is
// mma.sync.m16n8k4.f64 (measured at ~37 TFLOP/s on B200, the same rate as
// DFMA).  A CTA computes a BM x BN tile with WARPS_M x WARPS_N warps, each
// warp a (BM/WARPS_M) x (BN/WARPS_N) tile of 16x8 MMAs; K is streamed in
// chunks of BK through a STAGES-deep cp.async pipeline into padded shared
// tiles (A k-major with stride BM + 4, B n-major with stride BK + 4: both
// give conflict-free fragment loads); fragments are double-buffered in
// registers so shared-memory latency hides behind the previous k-step's MMAs.  The C tile is prefetched into L2 when
// the CTA starts so the read-modify-write of the epilogue hits L2.
// Accumulation is C - sum_k(a*b), the sum formed in FP64 by the tensor core.
#include <atomic>

#include "delayed_pivoting_b200.h"
#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace gemm {

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

template <int BM_, int BN_, int BK_, int STAGES_, int WARPS_M_, int WARPS_N_, int MINB_>
struct Cfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_, STAGES = STAGES_;
  static constexpr int WARPS_M = WARPS_M_, WARPS_N = WARPS_N_, MINB = MINB_;
  static constexpr int THREADS = 32 * WARPS_M * WARPS_N;
  static constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;  // warp tile
  static constexpr int MI = WTM / 16, NI = WTN / 8;
  // A fragments are read by half-warps of (g = 0..3, t = 0..3) at t*LDA_S + g:
  // LDA_S == 4 (mod 16) doubles puts the 16 lanes on 16 distinct 8-byte banks.
  static constexpr int LDA_S = BM + 4;
  static constexpr int LDB_S = BK + 4;  // == 4 (mod 16) doubles
  static constexpr int A_STAGE = BK * LDA_S;
  static constexpr int B_STAGE = BN * LDB_S;
  static constexpr size_t SMEM = (size_t)STAGES * (A_STAGE + B_STAGE) * sizeof(double);
  static_assert(BM % 16 == 0 && BN % 8 == 0 && WTM % 16 == 0 && WTN % 8 == 0, "tile");
  static_assert((BM * BK) % THREADS == 0 && (BN * BK) % THREADS == 0, "loader");
  static_assert(LDA_S % 16 == 4 && LDB_S % 16 == 4, "bank layout");
};

template <class C>
__global__ void __launch_bounds__(C::THREADS, C::MINB)
dgemm_minus_kernel(int M, int N, int K, const double* __restrict__ A, long long lda,
                   const double* __restrict__ B, long long ldb, double* Cm, long long ldc,
                   const int* gate, bool lower) {
  if (gate && *gate >= 0) return;  // an enqueued panel sequence stopped before this update
  extern __shared__ __align__(16) double gsm[];
  double* As = gsm;                         // [STAGES][BK][LDA_S]
  double* Bs = gsm + C::STAGES * C::A_STAGE;  // [STAGES][BN][LDB_S]

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp / C::WARPS_N, wn = warp % C::WARPS_N;
  const int g = lane >> 2, t = lane & 3;
  long long m0, n0;
  if (lower) {
    // Lower mode (M == N, C symmetric, its lower triangle only; BM == BN): a
    // 1-D grid over the tiles (bi, bj) with bj <= bi, t = bi (bi + 1) / 2 + bj.
    const long long t = blockIdx.x;
    long long bi = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
    while (bi * (bi + 1) / 2 > t) --bi;
    m0 = bi * C::BM;
    n0 = (t - bi * (bi + 1) / 2) * C::BN;
  } else {
    m0 = (long long)blockIdx.x * C::BM;
    n0 = (long long)blockIdx.y * C::BN;
  }

  // Prefetch this CTA's C tile into L2 (128-byte lines, in-bounds only).
  {
    const int rows = (int)min((long long)C::BM, M - m0);
    const int cols = (int)min((long long)C::BN, N - n0);
    const int lines_per_col = (rows * 8 + 127) / 128 + 1;
    for (int e = tid; e < cols * lines_per_col; e += C::THREADS) {
      const int c = e / lines_per_col, l = e % lines_per_col;
      const int r = min(rows - 1, l * 16);
      const double* p = Cm + idx(m0 + r, n0 + c, ldc);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  }

  const int ktiles = (K + C::BK - 1) / C::BK;

  auto load_stage = [&](int stage, int kt) {
    double* as = As + stage * C::A_STAGE;
    double* bs = Bs + stage * C::B_STAGE;
    const int k0 = kt * C::BK;
#pragma unroll
    for (int i = 0; i < (C::BM * C::BK) / C::THREADS; ++i) {
      const int e = tid + i * C::THREADS;
      const int r = e % C::BM, kk = e / C::BM;
      const bool ok = (m0 + r < M) && (k0 + kk < K);
      const double* src = ok ? A + idx(m0 + r, k0 + kk, lda) : A;
      cp_async8(as + kk * C::LDA_S + r, src, ok);
    }
#pragma unroll
    for (int i = 0; i < (C::BN * C::BK) / C::THREADS; ++i) {
      const int e = tid + i * C::THREADS;
      const int kk = e % C::BK, c = e / C::BK;
      const bool ok = (n0 + c < N) && (k0 + kk < K);
      const double* src = ok ? B + idx(k0 + kk, n0 + c, ldb) : B;
      cp_async8(bs + c * C::LDB_S + kk, src, ok);
    }
  };

  double acc[C::MI][C::NI][4];
#pragma unroll
  for (int i = 0; i < C::MI; ++i)
#pragma unroll
    for (int j = 0; j < C::NI; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

#pragma unroll
  for (int s = 0; s < C::STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<C::STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + C::STAGES - 1;
      if (nk < ktiles) load_stage(nk % C::STAGES, nk);
      cp_async_commit();
    }
    const double* as = As + (kt % C::STAGES) * C::A_STAGE;
    const double* bs = Bs + (kt % C::STAGES) * C::B_STAGE;
    double af[2][C::MI][2], bf[2][C::NI];
    auto load_frag = [&](int buf, int kk) {
#pragma unroll
      for (int mi = 0; mi < C::MI; ++mi) {
        const double* ap = as + (kk + t) * C::LDA_S + wm * C::WTM + mi * 16 + g;
        af[buf][mi][0] = ap[0];
        af[buf][mi][1] = ap[8];
      }
#pragma unroll
      for (int ni = 0; ni < C::NI; ++ni)
        bf[buf][ni] = bs[(wn * C::WTN + ni * 8 + g) * C::LDB_S + kk + t];
    };
    load_frag(0, 0);
#pragma unroll
    for (int kk = 0; kk < C::BK; kk += 4) {
      const int cur = (kk >> 2) & 1;
      if (kk + 4 < C::BK) load_frag(cur ^ 1, kk + 4);
#pragma unroll
      for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < C::NI; ++ni)
          mma_f64_16x8x4(acc[mi][ni], af[cur][mi][0], af[cur][mi][1], bf[cur][ni]);
    }
  }
  cp_async_wait<0>();

  // Epilogue: C -= acc, one 16-row block at a time with all its loads issued
  // before the first store.
#pragma unroll
  for (int mi = 0; mi < C::MI; ++mi) {
    double old[C::NI][4];
#pragma unroll
    for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const long long r = m0 + wm * C::WTM + mi * 16 + g + 8 * (v >> 1);
        const long long c = n0 + wn * C::WTN + ni * 8 + 2 * t + (v & 1);
        old[ni][v] = (r < M && c < N) ? Cm[idx(r, c, ldc)] : 0.0;
      }
#pragma unroll
    for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const long long r = m0 + wm * C::WTM + mi * 16 + g + 8 * (v >> 1);
        const long long c = n0 + wn * C::WTN + ni * 8 + 2 * t + (v & 1);
        if (r < M && c < N && (!lower || r >= c)) Cm[idx(r, c, ldc)] = old[ni][v] - acc[mi][ni][v];
      }
  }
}

template <class C>
void launch(int M, int N, int K, const double* A, long long lda, const double* B, long long ldb,
            double* Cm, long long ldc, cudaStream_t s, const int* gate, bool lower = false) {
  dp::ensure_smem((const void*)dgemm_minus_kernel<C>, C::SMEM);
  dim3 grid((M + C::BM - 1) / C::BM, (N + C::BN - 1) / C::BN);
  if (lower) {  // the lower-triangle tile grid needs square tiles
    if constexpr (C::BM == C::BN) {
      const unsigned nt = grid.x;
      grid = dim3(nt * (nt + 1) / 2);
    } else {
      return;
    }
  }
  dp::note_launch();
  dgemm_minus_kernel<C>
      <<<grid, C::THREADS, C::SMEM, s>>>(M, N, K, A, lda, B, ldb, Cm, ldc, gate, lower);
}

// 128 x 128 tiles, 8 warps of 64 x 32, one CTA per SM (212 KB of stages).
using Big = Cfg<128, 128, 32, 3, 2, 4, 1>;
// 128 x 64 tiles, 4 warps of 64 x 32, 16-deep k chunks in 4 stages (108 KB):
// two CTAs per SM, so one CTA's pipeline fill and C read-modify-write overlap
// the other's MMAs - with K = one outer block (256) those fixed costs are a
// large part of a 128 x 128 tile's life.
using Half = Cfg<128, 64, 16, 4, 2, 2, 2>;
// Few columns (the refinement residual B - A X, N = right-hand sides): 64 x 32
// tiles, 4 warps of 16 x 32, two CTAs per SM, so M / 64 CTAs stream A.
using Skinny = Cfg<64, 32, 32, 4, 4, 1, 2>;

// 64 x 64 tiles, 4 warps of 32 x 32, three CTAs per SM (57 KB of stages).
using Small = Cfg<64, 64, 16, 3, 2, 2, 3>;
// The same tile with two stages and four CTAs per SM (at most 128
// registers; 16 warps per SM hide the shallow pipeline): the fastest
// measured on B200 at every update shape of the LU, so the automatic choice.
// 16384 x 16384 updates: 29.6 TF/s at K = 256 and 24.2 at K = 64 (three-
// stage 64 x 64: 29.1 / 21.8; 128 x 64: 26.4 / 18.3; cuBLAS DGEMM 32.7 / 20.8).
using Small4 = Cfg<64, 64, 16, 2, 2, 2, 4>;
// 128 x 64 tiles as Half with 8 warps of 32 x 32: 16 warps per SM.
using HalfW8 = Cfg<128, 64, 16, 4, 4, 2, 2>;
// 64 x 128 tiles (the shape of the library DGEMM on this part), three stages
// of 16: 4 warps of 32 x 64, or 8 warps of 32 x 32; two CTAs per SM.
using Wide = Cfg<64, 128, 16, 3, 2, 2, 2>;
using Wide8 = Cfg<64, 128, 16, 3, 2, 4, 2>;
// 64 x 64 tiles with 32-deep k chunks in two stages, three CTAs per SM.
using SmallK32 = Cfg<64, 64, 32, 2, 2, 2, 3>;

// 0 automatic (Small4), 1 Big, 2 Half, 3 Small, 4 HalfW8, 5 Small4, 6 Wide,
// 7 Wide8, 8 SmallK32
std::atomic<int> g_tile{0};

}  // namespace gemm

// Every configuration accumulates each element over k in the same order
// (k = 0, 1, ... in chunks of 4, one accumulator), so the choice of tile
// changes no result bit.
void launch_gemm_minus(int M, int N, int K, const double* A, long long lda, const double* B,
                       long long ldb, double* C, long long ldc, cudaStream_t s, const int* gate) {
  if (M <= 0 || N <= 0 || K <= 0) return;
  const int tile = gemm::g_tile.load(std::memory_order_relaxed);
  if (N <= 32)
    gemm::launch<gemm::Skinny>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else if (tile == 1)
    gemm::launch<gemm::Big>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else if (tile == 2)
    gemm::launch<gemm::Half>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else if (tile == 3)
    gemm::launch<gemm::Small>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else if (tile == 4)
    gemm::launch<gemm::HalfW8>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else if (tile == 6)
    gemm::launch<gemm::Wide>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else if (tile == 7)
    gemm::launch<gemm::Wide8>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else if (tile == 8)
    gemm::launch<gemm::SmallK32>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
  else
    gemm::launch<gemm::Small4>(M, N, K, A, lda, B, ldb, C, ldc, s, gate);
}

// Lower triangle of the symmetric N x N block C -= A(N x K) * B(K x N), the
// strict upper triangle of C untouched (the LDL^T trailing update, where
// A B = L D L^T is symmetric); 64 x 64 tiles, only those on or below the
// diagonal launched.
void launch_gemm_minus_lower(int N, int K, const double* A, long long lda, const double* B,
                             long long ldb, double* C, long long ldc, cudaStream_t s) {
  if (N <= 0 || K <= 0) return;
  gemm::launch<gemm::Small4>(N, N, K, A, lda, B, ldb, C, ldc, s, nullptr, true);
}

}  // namespace dp

extern "C" {

int dp_schur_update_device(int M, int N, int K, const double* A, int lda, const double* B,
                           int ldb, double* C, int ldc, void* stream) {
  if (M < 0 || N < 0 || K < 0) return dp::kInvalidArgument;
  if (M == 0 || N == 0 || K == 0) return dp::kOk;
  if (!A || !B || !C || lda < M || ldb < K || ldc < M) return dp::kInvalidArgument;
  dp::launch_gemm_minus(M, N, K, A, lda, B, ldb, C, ldc, static_cast<cudaStream_t>(stream));
  return cudaGetLastError() == cudaSuccess ? dp::kOk : dp::kCudaFailure;
}

int dp_gemm_tile(int tile) {
  if (tile < 0 || tile > 8) return -1;
  return dp::gemm::g_tile.exchange(tile);
}

}  // extern "C"
