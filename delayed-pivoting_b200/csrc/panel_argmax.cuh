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

// D = A B + C on the FP64 tensor path, one 16 x 8 x 4 step (a0 = A(g, t),
// a1 = A(g + 8, t), b0 = B(t, g); c = C(g, 2t), C(g, 2t + 1), C(g + 8, 2t),
// C(g + 8, 2t + 1) with g = lane / 4, t = lane % 4).
__device__ __forceinline__ void mma_f64(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// ---- cluster exchange by transaction barriers ------------------------------
// A CTA expects a known number of bytes per exchange on a barrier in its own
// shared memory; its peers write them with st.async, each store completing
// its bytes on that barrier, so a reader waits for the data alone (one-way
// latency) instead of for every CTA of the cluster to reach a barrier.

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
// The address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ unsigned peer_addr(unsigned local, int rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
__device__ __forceinline__ void xbar_init(unsigned bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
// Makes initialised barriers visible to the cluster's other CTAs.
__device__ __forceinline__ void xbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// The one local arrival of a phase, announcing `bytes` to come.
__device__ __forceinline__ void xbar_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool xbar_test(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of parity `parity` to complete; false when
// kSpinLimitNs passed first.
__device__ __forceinline__ bool xbar_wait(unsigned bar, unsigned parity) {
  if (xbar_test(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i)
      if (xbar_test(bar, parity)) return true;
    if (globaltimer_ns() - t0 > kSpinLimitNs) return false;
  }
}
// 16 bytes to peer shared memory `peer` (a peer_addr), completing them on
// the peer's barrier `peer_bar`.
__device__ __forceinline__ void st_async16(unsigned peer, uint4 v, unsigned peer_bar) {
  asm volatile(
      "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];"
      ::"r"(peer), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(peer_bar)
      : "memory");
}
// The two halves of a cluster barrier: writes before arrive() are visible to
// every CTA of the cluster after its wait().
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

}  // namespace panel
}  // namespace dp
