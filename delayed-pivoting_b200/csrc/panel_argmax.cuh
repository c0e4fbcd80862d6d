// Warp-level pieces of the panel kernels' pivot search: the best (largest
// magnitude, then smallest row) candidate with its runner-up, reduced over a
// warp by bit-pattern maxima of non-negative magnitudes (NaN never enters:
// offer() skips it), and the asynchronous copies that stage a panel slice.
#pragma once

#include "dp_device.cuh"

namespace dp {
namespace panel {

struct __align__(16) LocalBest {
  double val;
  int row;     // local row, -1 when none
  int pad;
  double sec;  // largest magnitude among the other rows seen
};

// Offers magnitude v of local row r to a running (best, runner-up) pair.
// Equal magnitudes keep the earlier row (rows arrive in increasing order per
// thread) and make the runner-up equal to the best: an exact tie.
__device__ __forceinline__ void offer(LocalBest& b, double v, int r) {
  if (v > b.val) {
    b.sec = b.val;
    b.val = v;
    b.row = r;
  } else if (v > b.sec) {
    b.sec = v;
  }
}

// Largest of the lanes' non-negative magnitudes (bit-pattern order).
__device__ __forceinline__ double warp_max_pos(double v) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(u >> 32), lo = (unsigned)u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  return __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

// Best (largest magnitude, then smallest row) over the warp's lanes, every
// lane getting the result.  Magnitudes are >= 0 and a missing candidate
// offers (0, INT_MAX), so the bit patterns order like the values: max of the
// high word, of the low word among its holders, then min row - three warp
// reductions instead of five shuffle rounds.
__device__ __forceinline__ void warp_best(double v, int row, double& bv, int& brow) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(u >> 32), lo = (unsigned)u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const int key = (hi == mhi && lo == mlo) ? row : 0x7fffffff;
  brow = __reduce_min_sync(0xffffffffu, key);
  bv = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

// Best of the warp's (best, runner-up) pairs; the runner-up of the union is
// the largest of the winner lane's runner-up and every other lane's best.
__device__ __forceinline__ LocalBest warp_lb(LocalBest v) {
  double bv;
  int br;
  warp_best(v.row >= 0 ? v.val : 0.0, v.row >= 0 ? v.row : 0x7fffffff, bv, br);
  const bool win = v.row >= 0 && v.row == br;
  const double sec = warp_max_pos(win ? v.sec : (v.row >= 0 ? v.val : v.sec));
  return LocalBest{br == 0x7fffffff ? 0.0 : bv, br == 0x7fffffff ? -1 : br, 0, sec};
}

// 8-byte asynchronous global -> shared copy (L1-allocating), and the wait
// for every copy this thread issued.
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

}  // namespace panel
}  // namespace dp
