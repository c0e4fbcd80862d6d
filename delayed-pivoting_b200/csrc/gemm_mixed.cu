// Mixed-precision Schur-complement update on the 5th-generation tensor cores:
//   C(M x N, FP64) -= A(M x K, FP64) * B(K x N, FP64)
// with the product formed from a BF16 split of A and B into TERMS pieces
// (x = x1 + x2 [+ x3], each piece the BF16 rounding of what the earlier ones
// left) and the products whose pieces sum to at most TERMS - 1 ranks below
// the leading one:
//   TERMS = 2 (BF16x3):  A1B1 + A1B2 + A2B1                   (3 products)
//   TERMS = 3 (BF16x6):  A1B1 + A1B2 + A2B1 + A1B3 + A2B2 + A3B1  (6 products)
// accumulated in FP32 in tensor memory, then subtracted from C in FP64.
// This replaces the FP64 trailing update (delayed_lu/delayed_dgetrf.cpp:80-83)
// in the mixed-precision factorisation; pivot search, delay / fallback
// decisions and the panel stay in FP64.  Relative error of one update is about
// 2^-16 with three products and about 2^-24 (FP32 accumulation) with six;
// FP64 iterative refinement recovers full accuracy.
//
// Pipeline:
//   split_*_kernel  FP64 column-major -> BF16 pieces, K-major, K padded to 64
//   gemm kernel     persistent (one CTA per SM over 128 x 128 tiles of C),
//                   warp-specialised: a TMA warp feeds 128 x 64 BF16 boxes
//                   (128-byte swizzle) into a 2-stage ring, an MMA warp
//                   issues tcgen05.mma (kind::f16, FP32 accumulation) into a
//                   double-buffered TMEM accumulator, 16 epilogue warps
//                   prefetch their rows of C, then C -= acc in FP64 through
//                   tcgen05.ld while the next tile's MMAs run
// Every mbarrier wait is bounded; on timeout the kernel records
// kDeviceTimeout, skips the rest and still frees its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {

namespace mixed {

constexpr int BM = 128, BN = 128, BK = 64;  // BK: BF16 elements per 128-byte swizzle row
constexpr int kTileBytes = BM * BK * 2;     // 16 KB per operand tile (BN == BM)
constexpr int kStages = 2;
// A pieces then B pieces per stage
template <int TERMS>
constexpr int stage_bytes() { return 2 * TERMS * kTileBytes; }
template <int TERMS>
constexpr size_t smem_bytes() { return (size_t)kStages * stage_bytes<TERMS>() + 1024; }

// ---------------------------------------------------------------- split ----
template <int TERMS>
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 (&piece)[TERMS]) {
#pragma unroll
  for (int t = 0; t < TERMS; ++t) {
    piece[t] = __double2bfloat16(x);
    x -= (double)__bfloat162float(piece[t]);
  }
}

// A (M x K, column-major, lda) -> pieces [t][M][Kp] (K contiguous), piece t at
// out + t * M * Kp.  32x32 tiles transposed through shared memory so both
// sides stay coalesced.
template <int TERMS>
__global__ void split_a_kernel(const double* __restrict__ A, long long lda, int M, int K, int Kp,
                               __nv_bfloat16* __restrict__ out) {
  __shared__ double t[32][33];
  const int m0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int i = ty; i < 32; i += 8) {
    const int m = m0 + tx, k = k0 + i;
    t[i][tx] = (m < M && k < K) ? A[idx(m, k, lda)] : 0.0;
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int m = m0 + i, k = k0 + tx;
    if (m < M && k < Kp) {
      __nv_bfloat16 pc[TERMS];
      split_bf16<TERMS>(t[tx][i], pc);
#pragma unroll
      for (int q = 0; q < TERMS; ++q) out[(size_t)q * M * Kp + (size_t)m * Kp + k] = pc[q];
    }
  }
}

// B (K x N, column-major, ldb) -> pieces [t][N][Kp] (K contiguous).
template <int TERMS>
__global__ void split_b_kernel(const double* __restrict__ B, long long ldb, int K, int N, int Kp,
                               __nv_bfloat16* __restrict__ out) {
  const long long total = (long long)N * Kp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(e / Kp), k = (int)(e - (long long)n * Kp);
    const double x = k < K ? B[idx(k, n, ldb)] : 0.0;
    __nv_bfloat16 pc[TERMS];
    split_bf16<TERMS>(x, pc);
#pragma unroll
    for (int q = 0; q < TERMS; ++q) out[(size_t)q * total + e] = pc[q];
  }
}

// ------------------------------------------------------ PTX wrappers ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const uint32_t addr = smem_u32(bar);
  const unsigned long long t0 = globaltimer_ns();
  for (unsigned it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 255u) == 255u && globaltimer_ns() - t0 > kSpinLimitNs) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, uint64_t* bar, int x,
                                            int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand
// tile (8-row x 128-byte swizzle atoms, atoms 1024 bytes apart).
__device__ __forceinline__ uint64_t umma_desc_k_sw128(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;          // start address (16-byte units)
  d |= 1ull << 16;                        // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset: next 8-row group
  d |= 1ull << 46;                        // descriptor version (sm_100)
  d |= 2ull << 61;                        // layout: 128-byte swizzle
  return d;
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = 128.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15},"
      " [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// -------------------------------------------------------------- GEMM ----
struct Maps {
  CUtensorMap a[3], b[3];
};

// Persistent, warp-specialised kernel: CTA c takes the 128 x 128 tiles c,
// c + grid, ... of C (m fastest).
//   warp 0 (one lane)  TMA producer: per K chunk of 64 the TERMS pieces of A
//                      and of B into a kStages ring (full / empty barriers)
//   warp 1 (one lane)  MMA issuer: tcgen05.mma of the split products into
//                      one of two 128-column TMEM accumulators (tile parity),
//                      tcgen05.commit frees a stage and, after the last
//                      chunk, hands the accumulator to the epilogue
//   warps 2..17        epilogue: each thread owns one row and 32 columns of
//                      the tile; it loads those 32 C values BEFORE the
//                      accumulator is ready (the FP64 read-modify-write of C
//                      is the bound: 16 bytes per element against 2 K x
//                      products flops), then C -= acc through tcgen05.ld
//                      and releases the accumulator - so the C traffic of
//                      tile t overlaps the MMAs of tile t + 1
// Warp w reads TMEM lanes 32 (w % 4) .. + 31 (the hardware's lane split);
// warps w, w + 4, w + 8, w + 12 take the four 32-column quarters of those
// rows.
constexpr int kEpiWarps = 16;
constexpr int kThreadsP = 64 + 32 * kEpiWarps;  // 576
constexpr int kEpiCols = BN / (kEpiWarps / 4);  // 32 columns per epilogue thread
constexpr unsigned kTmemColsP = 2 * BN;         // double-buffered accumulator

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int TERMS>
__global__ void __launch_bounds__(kThreadsP, 1)
gemm_bf16x3_kernel(const __grid_constant__ Maps tm, int M, int N, int kchunks, double* C,
                   long long ldc, int* status) {
  constexpr int kStageBytes = stage_bytes<TERMS>();
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages];
  __shared__ __align__(8) uint64_t tfull_bar[2], tempty_bar[2], done_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int failed;
  unsigned char* smem =
      reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_m = (M + BM - 1) / BM;
  const int tiles = tiles_m * ((N + BN - 1) / BN);

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_sh)),
                 "r"(kTmemColsP)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], kEpiWarps);
    }
    mbar_init(&done_bar, 1);
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;
  // `failed` is written and polled by different warps: volatile accesses
  volatile int* const vfailed = &failed;
  auto fail = [&] {
    *vfailed = 1;
    atomicCAS(status, kOk, kDeviceTimeout);
  };

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int g = 0;      // chunk counter over this CTA's tiles
      for (int t = blockIdx.x; t < tiles && !*vfailed; t += gridDim.x) {
        const int m0 = (t % tiles_m) * BM, n0 = (t / tiles_m) * BN;
        for (int c = 0; c < kchunks; ++c, ++g) {
          const int s = g % kStages;
          const unsigned ph = (unsigned)((g / kStages) & 1);
          if (!mbar_wait(&empty_bar[s], ph ^ 1u)) {  // a fresh barrier passes parity 1
            fail();
            break;
          }
          unsigned char* st = smem + (size_t)s * kStageBytes;
          mbar_expect_tx(&full_bar[s], kStageBytes);
#pragma unroll
          for (int q = 0; q < TERMS; ++q) {
            tma_load_2d(st + q * kTileBytes, &tm.a[q], &full_bar[s], c * BK, m0);
            tma_load_2d(st + (TERMS + q) * kTileBytes, &tm.b[q], &full_bar[s], c * BK, n0);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      const uint32_t idesc = idesc_bf16_f32(BM, BN);
      int g = 0, it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++it) {
        const int buf = it & 1;
        if (!mbar_wait(&tempty_bar[buf], (unsigned)((it >> 1) & 1) ^ 1u)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(buf * BN);
        for (int c = 0; c < kchunks; ++c, ++g) {
          const int s = g % kStages;
          const unsigned ph = (unsigned)((g / kStages) & 1);
          if (!mbar_wait(&full_bar[s], ph)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          unsigned char* st = smem + (size_t)s * kStageBytes;
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            uint64_t ad[TERMS], bd[TERMS];
#pragma unroll
            for (int q = 0; q < TERMS; ++q) {
              ad[q] = umma_desc_k_sw128(st + q * kTileBytes + kk * 32);
              bd[q] = umma_desc_k_sw128(st + (TERMS + q) * kTileBytes + kk * 32);
            }
            // products of pieces (i, j) with i + j <= TERMS - 1, leading one first
            bool first = c == 0 && kk == 0;
#pragma unroll
            for (int d = 0; d < TERMS; ++d)
#pragma unroll
              for (int i = 0; i <= d; ++i) {
                umma_f16(acc, ad[i], bd[d - i], idesc, first ? 0u : 1u);
                first = false;
              }
          }
          umma_commit(&empty_bar[s]);  // the stage is free once these MMAs complete
        }
        if (!ok) break;
        umma_commit(&tfull_bar[buf]);  // the accumulator is complete
      }
      if (!ok) fail();
      umma_commit(&done_bar);  // arrives once every issued MMA has completed
    }
  } else {  // epilogue
    const int q = warp & 3, h = (warp - 2) >> 2;
    const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
    int it = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
      const int buf = it & 1;
      const int m0 = (t % tiles_m) * BM, n0 = (t / tiles_m) * BN;
      const int row = m0 + q * 32 + lane;
      const int col0 = n0 + h * kEpiCols;
      const bool row_ok = row < M;
      double* crow = C + idx(row_ok ? row : 0, col0, ldc);
      double old[kEpiCols];  // read-only, L2-cached loads: all in flight at once
#pragma unroll
      for (int j = 0; j < kEpiCols; ++j)
        old[j] = (row_ok && col0 + j < N) ? __ldcg(crow + (size_t)j * ldc) : 0.0;
      const bool got = mbar_wait(&tfull_bar[buf], (unsigned)((it >> 1) & 1));
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (!got || *vfailed) {
        if (lane == 0) fail();
        break;
      }
      const uint32_t acc = lane_base + (uint32_t)(buf * BN + h * kEpiCols);
#pragma unroll
      for (int cc = 0; cc < kEpiCols / 16; ++cc) {
        uint32_t r[16];
        tmem_ld16(acc + (uint32_t)(cc * 16), r);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int jj = cc * 16 + j;
          if (row_ok && col0 + jj < N)
            crow[(size_t)jj * ldc] = old[jj] - (double)__uint_as_float(r[j]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty_bar[buf]);
    }
  }
  // every issued MMA has completed before the tensor memory is released
  __syncthreads();
  if (warp == 1) {
    const bool ok = mbar_wait(&done_bar, 0);
    if (!ok && lane == 0) fail();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemColsP)
                 : "memory");
  }
}

// ------------------------------------------------------ host helpers ----
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 2-D BF16 tensor [rows][kp] (kp contiguous), box 64 x 128, 128-byte swizzle.
bool make_map(CUtensorMap* tm, void* base, int rows, int kp) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)BM};
  cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace mixed

size_t mixed_scratch_bytes(int max_rows, int max_cols, int max_k, int terms) {
  const size_t kp = (size_t)((max_k + mixed::BK - 1) / mixed::BK) * mixed::BK;
  return (size_t)terms * ((size_t)max_rows + (size_t)max_cols) * kp * sizeof(__nv_bfloat16) + 4096;
}

namespace mixed {

// CTAs of the tensor-core update (dp_mixed_gemm_grid): 0 automatic = one
// per tile (an SM frees as soon as its tile is done, so the panel stream's
// clusters, waiting for whole SMs, start sooner: a mixed n = 16384 LU took
// 78.6 ms against 89.1 with one persistent CTA per SM), g > 0 at most g, -1
// one per SM (persistent over the tiles).
std::atomic<int> g_grid{0};

template <int TERMS>
int launch(int M, int N, int K, const double* A, long long lda, const double* B, long long ldb,
           double* C, long long ldc, void* scratch, int* status, cudaStream_t s) {
  if (!ensure_smem((const void*)gemm_bf16x3_kernel<TERMS>, smem_bytes<TERMS>()))
    return kCudaFailure;
  const int kp = (K + BK - 1) / BK * BK;
  auto* ap = reinterpret_cast<__nv_bfloat16*>(scratch);  // [TERMS][M][kp]
  auto* bp = ap + (size_t)TERMS * M * kp;                 // [TERMS][N][kp]
  dp::note_launch();
  split_a_kernel<TERMS><<<dim3((M + 31) / 32, (kp + 31) / 32), dim3(32, 8), 0, s>>>(A, lda, M, K,
                                                                                  kp, ap);
  {
    const long long total = (long long)N * kp;
    long long grid = (total + 255) / 256;
    if (grid > 148 * 16) grid = 148 * 16;
    dp::note_launch();
    split_b_kernel<TERMS><<<(int)grid, 256, 0, s>>>(B, ldb, K, N, kp, bp);
  }
  Maps tm;
  for (int q = 0; q < TERMS; ++q)
    if (!make_map(&tm.a[q], ap + (size_t)q * M * kp, M, kp) ||
        !make_map(&tm.b[q], bp + (size_t)q * N * kp, N, kp))
      return kLibraryFailure;
  const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  const int gp = g_grid.load(std::memory_order_relaxed);
  const int cap = gp == 0 ? tiles : gp < 0 ? sm_count() : gp;
  const int grid = std::max(1, std::min(tiles, cap));
  dp::note_launch();
  gemm_bf16x3_kernel<TERMS><<<grid, kThreadsP, smem_bytes<TERMS>(), s>>>(tm, M, N, kp / BK, C, ldc,
                                                                        status);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

}  // namespace mixed

// C(M x N) -= A(M x K) * B(K x N) through the BF16 split tensor-core path
// with `terms` pieces (2: three products, 3: six products).  scratch must
// hold mixed_scratch_bytes(M, N, K, terms) bytes (256-byte aligned).
int launch_gemm_minus_mixed(int M, int N, int K, const double* A, long long lda, const double* B,
                            long long ldb, double* C, long long ldc, void* scratch, int terms,
                            int* status, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return kOk;
  if (terms == 3) return mixed::launch<3>(M, N, K, A, lda, B, ldb, C, ldc, scratch, status, s);
  return mixed::launch<2>(M, N, K, A, lda, B, ldb, C, ldc, scratch, status, s);
}

}  // namespace dp

// The mixed-precision update alone (tests and measurements of the kernel):
// scratch from the stream-ordered pool, status read back (synchronises).
extern "C" int dp_schur_update_mixed_device(int M, int N, int K, const double* A, int lda,
                                            const double* B, int ldb, double* C, int ldc,
                                            int precision, void* stream) {
  using namespace dp;
  const int terms = mixed_terms(precision);
  if (M < 0 || N < 0 || K < 0 || terms == 0) return kInvalidArgument;
  if (M == 0 || N == 0 || K == 0) return kOk;
  if (!A || !B || !C || lda < M || ldb < K || ldc < M) return kInvalidArgument;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t bytes = mixed_scratch_bytes(M, N, K, terms) + 256;
  char* scratch = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&scratch), bytes, st) != cudaSuccess) {
    cudaGetLastError();
    return kAllocationFailed;
  }
  int* status = reinterpret_cast<int*>(scratch + bytes - 256);
  int rc = cudaMemsetAsync(status, 0, sizeof(int), st) == cudaSuccess ? kOk : kCudaFailure;
  if (rc == kOk)
    rc = launch_gemm_minus_mixed(M, N, K, A, lda, B, ldb, C, ldc, scratch, terms, status, st);
  int h = kOk;
  if (rc == kOk &&
      (cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess))
    rc = kCudaFailure;
  cudaFreeAsync(scratch, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == kOk) rc = kCudaFailure;
  if (rc != kOk) cudaGetLastError();
  return rc == kOk ? h : rc;
}

extern "C" int dp_mixed_gemm_grid(int policy) {
  if (policy < -1 || policy > 65536) return -2;
  return dp::mixed::g_grid.exchange(policy);
}
