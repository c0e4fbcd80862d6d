// Triangular solves with many right-hand sides in ONE launch (the solve and
// refinement path: getrs and every refinement correction).
//
// Y (n x nrhs, nrhs <= 64) <- T^{-1} Y with T the unit-lower L or the upper U
// (with its diagonal) of a compact L\U factorisation.  The rows are cut into
// blocks of 64; a grid of up to one CTA per SM takes the blocks in dependency order
// (lower: top down, upper: bottom up) by tickets from an atomic counter, so
// every block a CTA waits for was claimed earlier by a CTA that is already
// running: the earliest unfinished block always has every input it needs,
// and no CTA depends on one that has not started - no co-residency (no
// cooperative launch) is needed, and the launch starts on whatever SMs are
// free.  A block
//   1. starts from its rows of Y,
//   2. for each earlier block j: waits until j is published (a flag set to the
//      launch's epoch, read with acquire semantics, bounded by kSpinLimitNs),
//      stages y_j in shared memory and subtracts T(i, j) y_j; T(i, j) arrives
//      by asynchronous copies issued one block ahead (T read once),
//   3. multiplies by the inverse of its 64 x 64 diagonal block (inverses made
//      once per factorisation by diag_inverse_kernel, staged in shared memory
//      while the dependencies were awaited) - a product over all threads
//      instead of a 64-step serial substitution on the critical path,
//   4. writes y_i and publishes it (fence, then a release store of the flag).
// A wait that runs out sets *status = kDeviceTimeout and every CTA returns.
#include <algorithm>
#include <atomic>

#include "dp_device.cuh"
#include "dp_kernels.h"

namespace dp {
namespace {

constexpr int kTB = 64;           // rows per block
constexpr int kTT = 256;          // threads
constexpr int kTRhs = 64;         // right-hand sides per launch
constexpr int kTAcc = kTRhs / 4;  // accumulators per thread (4 column groups)
constexpr int kTMaxGrid = 32;     // CTAs of one launch under a block-count policy

// CTAs of a launch (dp_tri_solve_grid): 0 -> min(blocks, SMs); g > 0 ->
// min(blocks, g); g < 0 -> one CTA per -g row blocks (at most kTMaxGrid).
std::atomic<int> g_tri_grid{0};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// T(r0 + k, c0 + c) for k, c < 64 into sm[c * kTB + k] (zeros outside the
// rows x cols block), 8-byte asynchronous copies.
__device__ __forceinline__ void stage_block(double* sm, const double* T, long long ldt, int r0,
                                            int c0, int rows, int cols) {
  for (int e = threadIdx.x; e < kTB * kTB; e += kTT) {
    const int k = e & (kTB - 1), c = e >> 6;
    if (k < rows && c < cols)
      cp_async8(sm + e, T + (r0 + k) + (long long)(c0 + c) * ldt);
    else
      sm[e] = 0.0;
  }
}

// inv + 2 * kTB * kTB * i holds, column-major, the inverse of the unit-lower
// L(i, i) then the inverse of the upper U(i, i) of diagonal block i (identity
// where the last block is shorter than kTB).  Warp w inverts columns w, w + 8,
// ... by substitution on the unit vectors, two rows per lane.
__global__ void __launch_bounds__(kTT) diag_inverse_kernel(const double* __restrict__ T,
                                                           long long ldt, int n, double* inv) {
  __shared__ double dg[kTB * kTB];
  const int i = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = i * kTB, rows = min(kTB, n - r0);
  for (int e = tid; e < kTB * kTB; e += kTT) {
    const int k = e & (kTB - 1), c = e >> 6;
    dg[e] = (k < rows && c < rows) ? T[(r0 + k) + (long long)(r0 + c) * ldt] : 0.0;
  }
  __syncthreads();
  double* Li = inv + (size_t)2 * kTB * kTB * i;
  double* Ui = Li + kTB * kTB;
  double v0[8], v1[8];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int c = warp + 8 * m;
    v0[m] = lane == c ? 1.0 : 0.0;
    v1[m] = lane + 32 == c ? 1.0 : 0.0;
  }
  for (int k = 0; k < rows - 1; ++k) {
    const double l0 = lane > k ? dg[k * kTB + lane] : 0.0;
    const double l1 = lane + 32 > k ? dg[k * kTB + lane + 32] : 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const double yk = __shfl_sync(0xffffffffu, k < 32 ? v0[m] : v1[m], k & 31);
      v0[m] = fma(-l0, yk, v0[m]);
      v1[m] = fma(-l1, yk, v1[m]);
    }
  }
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int c = warp + 8 * m;
    Li[c * kTB + lane] = v0[m];
    Li[c * kTB + lane + 32] = v1[m];
    v0[m] = lane == c ? 1.0 : 0.0;
    v1[m] = lane + 32 == c ? 1.0 : 0.0;
  }
  const double inv0 = lane < rows ? 1.0 / dg[lane * kTB + lane] : 1.0;
  const double inv1 = lane + 32 < rows ? 1.0 / dg[(lane + 32) * kTB + lane + 32] : 1.0;
  for (int k = rows - 1; k >= 0; --k) {
    const double u0 = lane < k ? dg[k * kTB + lane] : 0.0;
    const double u1 = lane + 32 < k ? dg[k * kTB + lane + 32] : 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if (k < 32) {
        if (lane == k) v0[m] *= inv0;
      } else {
        if (lane == k - 32) v1[m] *= inv1;
      }
      const double yk = __shfl_sync(0xffffffffu, k < 32 ? v0[m] : v1[m], k & 31);
      v0[m] = fma(-u0, yk, v0[m]);
      v1[m] = fma(-u1, yk, v1[m]);
    }
  }
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int c = warp + 8 * m;
    Ui[c * kTB + lane] = v0[m];
    Ui[c * kTB + lane + 32] = v1[m];
  }
}

__device__ __forceinline__ void cp_async16(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// MACC accumulators per thread: columns cg, cg + 4, ..., cg + 4 (MACC - 1)
// (nrhs <= 4 MACC), so a launch with few right-hand sides issues no idle FMAs.
template <bool kUpper, int MACC>
__global__ void __launch_bounds__(kTT, 1) tri_solve_kernel(const double* __restrict__ T,
                                                           long long ldt, int n,
                                                           const double* __restrict__ inv,
                                                           double* Y, long long ldy, int nrhs,
                                                           unsigned* flags, unsigned epoch,
                                                           int* status) {
  constexpr int kNp = MACC == 1 ? 4 : 1;  // partial sums per accumulator
  extern __shared__ double tsm[];
  double* ys = tsm;                  // y_j, [kTRhs][kTB]
  double* ds = ys + kTB * kTRhs;     // the block's right-hand sides, [kTRhs][kTB]
  double* dg = ds + kTB * kTRhs;     // diagonal block T(i, i), [kTB][kTB] column-major
  double* ls = dg + kTB * kTB;       // T(i, j) double buffer, 2 x [kTB][kTB]
  __shared__ int abort_all, ticket;
  const int tid = threadIdx.x, r = tid & (kTB - 1), cg = tid >> 6;
  const int nblk = (n + kTB - 1) / kTB;
  int* const counter = reinterpret_cast<int*>(flags + nblk);  // zeroed before the launch
  if (tid == 0) abort_all = 0;
  for (;;) {
    if (tid == 0) ticket = atomicAdd(counter, 1);
    __syncthreads();
    const int q = ticket;
    __syncthreads();  // every thread holds q before the next claim
    if (q >= nblk || abort_all) break;
    const int i = kUpper ? nblk - 1 - q : q;
    const int r0 = i * kTB, rows = min(kTB, n - r0);
    const int deps = kUpper ? nblk - 1 - i : i;
    // the diagonal block and the first off-diagonal block, in flight while
    // the dependencies are awaited
    {
      const double* src = inv + (size_t)2 * kTB * kTB * i + (kUpper ? kTB * kTB : 0);
      for (int e = 2 * tid; e < kTB * kTB; e += 2 * kTT) cp_async16(dg + e, src + e);
    }
    cp_async_commit();
    auto dep = [&](int t) { return kUpper ? nblk - 1 - t : t; };
    if (deps > 0) {
      const int j = dep(0);
      stage_block(ls, T, ldt, r0, j * kTB, rows, min(kTB, n - j * kTB));
    }
    cp_async_commit();
    double acc[MACC];
#pragma unroll
    for (int m = 0; m < MACC; ++m) {
      const int c = cg + 4 * m;
      acc[m] = (r < rows && c < nrhs) ? Y[(r0 + r) + c * ldy] : 0.0;
    }
    // thread 0 confirms block dep(t) before the barrier that opens step t
    auto await_dep = [&](int t) {
      if (tid != 0 || abort_all) return;
      const int j = dep(t);
      const unsigned long long t0 = globaltimer_ns();
      while (ld_acquire_u32(flags + j) != epoch) {
        if (globaltimer_ns() - t0 > kSpinLimitNs) {
          abort_all = 1;
          atomicExch(status, kDeviceTimeout);
          break;
        }
      }
    };
    if (deps > 0) await_dep(0);
    __syncthreads();
    for (int t = 0; t < deps; ++t) {
      if (abort_all) {
        cp_async_wait<0>();
        return;
      }
      const int j = dep(t);
      const int rj = j * kTB, rowsj = min(kTB, n - rj);
      double* lb = ls + (t & 1) * kTB * kTB;
      if (t + 1 < deps) {  // the next block's T(i, j') behind this one
        const int jn = dep(t + 1);
        stage_block(ls + ((t + 1) & 1) * kTB * kTB, T, ldt, r0, jn * kTB, rows,
                    min(kTB, n - jn * kTB));
      }
      cp_async_commit();
      for (int e = tid; e < kTB * nrhs; e += kTT) {
        const int k = e & (kTB - 1), c = e >> 6;
        ys[e] = k < rowsj ? __ldcg(Y + (rj + k) + c * ldy) : 0.0;
      }
      cp_async_wait<1>();  // lb has landed (the newest group may still be in flight)
      __syncthreads();
      if (r < rows) {
        // kNp interleaved partial sums (few right-hand sides: the per-thread
        // FMA chain, not the issue rate, bounds this step)
        double part[kNp][MACC];  // part[0] unused: the first sum is acc
#pragma unroll
        for (int q = 0; q < kNp; ++q)
#pragma unroll
          for (int m = 0; m < MACC; ++m) part[q][m] = 0.0;
#pragma unroll 8
        for (int k = 0; k < kTB; k += kNp) {
#pragma unroll
          for (int q = 0; q < kNp; ++q) {
            const double l = lb[(k + q) * kTB + r];
#pragma unroll
            for (int m = 0; m < MACC; ++m)
              if (cg + 4 * m < nrhs) {
                double& dst = q == 0 ? acc[m] : part[q][m];
                dst = fma(-l, ys[(cg + 4 * m) * kTB + k + q], dst);
              }
          }
        }
#pragma unroll
        for (int m = 0; m < MACC; ++m)
#pragma unroll
          for (int q = 1; q < kNp; ++q) acc[m] += part[q][m];
      }
      if (t + 1 < deps) await_dep(t + 1);
      __syncthreads();  // ys and lb are free; the next dependency is confirmed
    }
    cp_async_wait<0>();
#pragma unroll
    for (int m = 0; m < MACC; ++m) {
      const int c = cg + 4 * m;
      if (c < nrhs) ds[c * kTB + r] = acc[m];
    }
    __syncthreads();
    // y_i = inverse(T(i, i)) * (right-hand sides): thread (r, cg) forms rows
    // r of its columns
    if (r < rows) {
      double y[MACC], yp[kNp][MACC];  // yp[0] unused: the first sum is y
#pragma unroll
      for (int m = 0; m < MACC; ++m) {
        y[m] = 0.0;
#pragma unroll
        for (int q = 0; q < kNp; ++q) yp[q][m] = 0.0;
      }
#pragma unroll 8
      for (int k = 0; k < kTB; k += kNp) {
#pragma unroll
        for (int q = 0; q < kNp; ++q) {
          const double a = dg[(k + q) * kTB + r];
#pragma unroll
          for (int m = 0; m < MACC; ++m)
            if (cg + 4 * m < nrhs) {
              double& dst = q == 0 ? y[m] : yp[q][m];
              dst = fma(a, ds[(cg + 4 * m) * kTB + k + q], dst);
            }
        }
      }
#pragma unroll
      for (int m = 0; m < MACC; ++m)
#pragma unroll
        for (int q = 1; q < kNp; ++q) y[m] += yp[q][m];
#pragma unroll
      for (int m = 0; m < MACC; ++m) {
        const int c = cg + 4 * m;
        if (c < nrhs) Y[(r0 + r) + c * ldy] = y[m];
      }
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      st_release_u32(flags + i, epoch);
    }
  }
}

template <bool kUpper, int MACC>
int launch_tri(const double* T, long long ldt, int n, const double* inv, double* Y,
               long long ldy, int nrhs, unsigned* flags, unsigned epoch, int* status,
               cudaStream_t st) {
  const size_t smem = sizeof(double) * (2 * kTB * kTRhs + 3 * kTB * kTB);
  if (!ensure_smem((const void*)tri_solve_kernel<kUpper, MACC>, smem)) return kCudaFailure;
  const int sms = sm_count();
  const int per_sm = occupancy_once((const void*)tri_solve_kernel<kUpper, MACC>, kTT, smem);
  if (sms < 1 || per_sm < 1) return kCudaFailure;
  // Besides the chain of diagonal blocks, block i subtracts all i blocks
  // before it, T(i, 0:i) y(0:i): that work (the triangle, read once) spreads
  // over the CTAs, so one CTA per SM is the default - measured against 32
  // CTAs: n = 16384, one right-hand side, 2.6 ms against 6.1 per solve;
  // n = 8192 1.06 against 1.80; n = 4096 0.56 against 0.67.
  const int nblk = (n + kTB - 1) / kTB;
  const int policy = g_tri_grid.load(std::memory_order_relaxed);
  const int want = policy == 0 ? sms
                   : policy > 0 ? policy
                                : std::max(1, std::min(kTMaxGrid, (nblk - policy - 1) / -policy));
  const int grid = std::max(1, std::min(std::min(nblk, want), sms * per_sm));
  // the ticket counter after the block flags
  if (cudaMemsetAsync(flags + nblk, 0, sizeof(unsigned), st) != cudaSuccess) return kCudaFailure;
  note_launch();
  tri_solve_kernel<kUpper, MACC><<<grid, kTT, smem, st>>>(T, ldt, n, inv, Y, ldy, nrhs, flags,
                                                          epoch, status);
  if (cudaGetLastError() != cudaSuccess) return kCudaFailure;
  return kOk;
}

}  // namespace

int tri_solve_rhs_max() { return kTRhs; }
int tri_solve_flag_count(int n) { return (n + kTB - 1) / kTB + 1; }  // block flags, ticket
size_t tri_inverse_doubles(int n) { return (size_t)2 * kTB * kTB * ((n + kTB - 1) / kTB); }

int launch_diag_inverse(const double* lu, long long ldlu, int n, double* inv, cudaStream_t st) {
  if (n <= 0) return kOk;
  note_launch();
  diag_inverse_kernel<<<(n + kTB - 1) / kTB, kTT, 0, st>>>(lu, ldlu, n, inv);
  return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

int launch_tri_lower_unit(const double* L, long long ldl, int n, const double* inv, double* Y,
                          long long ldy, int nrhs, unsigned* flags, unsigned epoch, int* status,
                          cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return kOk;
  if (nrhs > kTRhs) return kInvalidArgument;
  if (nrhs <= 4) return launch_tri<false, 1>(L, ldl, n, inv, Y, ldy, nrhs, flags, epoch, status, st);
  if (nrhs <= 16) return launch_tri<false, 4>(L, ldl, n, inv, Y, ldy, nrhs, flags, epoch, status, st);
  return launch_tri<false, kTAcc>(L, ldl, n, inv, Y, ldy, nrhs, flags, epoch, status, st);
}

int launch_tri_upper(const double* U, long long ldu, int n, const double* inv, double* Y,
                     long long ldy, int nrhs, unsigned* flags, unsigned epoch, int* status,
                     cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return kOk;
  if (nrhs > kTRhs) return kInvalidArgument;
  if (nrhs <= 4) return launch_tri<true, 1>(U, ldu, n, inv, Y, ldy, nrhs, flags, epoch, status, st);
  if (nrhs <= 16) return launch_tri<true, 4>(U, ldu, n, inv, Y, ldy, nrhs, flags, epoch, status, st);
  return launch_tri<true, kTAcc>(U, ldu, n, inv, Y, ldy, nrhs, flags, epoch, status, st);
}

}  // namespace dp

extern "C" int dp_tri_solve_grid(int policy) {
  if (policy > 1024 || policy < -1024) return -2000;
  return dp::g_tri_grid.exchange(policy);
}
