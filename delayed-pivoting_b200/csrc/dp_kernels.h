// Kernel parameter blocks and host-side launch wrappers of the
// delayed-pivoting LU.  Internal to the library (not part of the C ABI).
#pragma once
#include <vector>

#include <cuda_runtime.h>

#include "delayed_pivoting_b200.h"
#include "dp_device.cuh"

namespace dp {

struct PanelParams {
  double* a;
  long long lda;
  int m;
  int begin, end;     // panel columns [begin, end), rows [begin, m)
  int rows_per_cta;   // R
  int positioned;     // pivot of the first step already sits at (begin, begin)
  int parity;         // which of the two slot buffers this launch uses
  int max_ctas;       // slot buffer stride
  int w_max;          // row-data buffer stride - 1
  double threshold;
  int* ipiv;          // device swap history (global step index)
  State* state;
  unsigned long long* slots;  // mailboxes [2][4][max_ctas reader][max_ctas writer][2 words]
  double* xdata;              // [4][max_ctas][w_max + 1]
  double* rowk;               // [4][w_max + 1]
  int* swap_block;            // [end - begin]: source row of block row begin + i
  int* swap_extra;            // [2 * (end - begin)]: (dst, src) pairs below `end`
  int gated;                  // cluster kernel: 1 -> do nothing when state->stop_k >= 0 (an
                              // earlier panel of the same enqueued sequence stopped)
};

__global__ void panel_factor_kernel(PanelParams p);
// Cluster variant: one thread-block cluster of C <= 16 CTAs holds the panel
// in distributed shared memory (launched with a cluster dimension).
__global__ void panel_cluster_kernel(PanelParams p);
size_t panel_cluster_smem_bytes(int w, int rows_per_cta);
// Cluster variant with the sub-panel in registers (panel_reg.cu), for up to
// panel_reg_max_rows() rows per CTA: the kernel instance for R rows per CTA
// (nullptr beyond the limit) and its dynamic shared memory.
int panel_reg_max_rows();
const void* panel_reg_kernel_for(int rows_per_cta);
size_t panel_reg_smem_bytes(int w, int rows_per_cta);
int panel_cluster_threads();
constexpr int kPanelThreadsHost = 256;
// Single-CTA panel (batched.cu) for panels of at most panel_small_max_rows()
// rows and panel_small_max_width() columns: same contract as the cluster
// panel, rows register-resident, one CTA barrier per step.
int panel_small_max_rows();
int panel_small_max_width();
int launch_panel_small(const PanelParams& pp, cudaStream_t st);
// x[0..len) <- seeded N(0,1) (hashed Box-Muller; tuner inputs).
void launch_fill_normal(double* x, long long len, unsigned long long seed, cudaStream_t st);
size_t panel_smem_bytes(int w, int rows_per_cta);

// Applies the composite row permutation of one panel (swap list written by
// panel_factor_kernel) to columns [c0, c1) and [c2, c3).  gate_begin >= 0:
// do nothing when state->stop_k is in [0, gate_begin) (a panel before this
// one stopped; its own stop, at or after gate_begin, still applies).
// [s0, s1) within [c2, c3): when no panel stopped (state->stop_k < 0) and the
// panel is at most laswp_solve_max_width() wide, also solve the panel's block
// rows of those columns with its unit lower triangle (U12 = L11^{-1} A12).
int laswp_solve_max_width();
void launch_laswp(double* a, long long lda, int begin, int nblock, const int* swap_block,
                  const int* swap_extra, const State* state, int c0, int c1, int c2, int c3,
                  cudaStream_t s, int gate_begin = -1, int s0 = 0, int s1 = 0);

// Swap lists of up to kSwapSeqLists consecutive panels (kSwapSeqEntries
// entries in all) applied in order by one launch of laswp_seq_kernel.
constexpr int kSwapSeqLists = 64;
constexpr int kSwapSeqEntries = 2048;
struct SwapSeq {
  int lists;
  int base;  // first row of the first panel
  int width[kSwapSeqLists];
};

// Applies the swap lists of `lists` consecutive panels starting at row
// `base` (panel p of width widths[p], its block part at blk[begin_p - base],
// up to widths[p] extra pairs at ext[2 (begin_p - base)], the unused ones
// holding a negative destination) to the columns [c0, c1) and [c2, c3), in
// panel order.  Returns the number of launches, or -1 when a panel is wider
// than the kernel's lists.
int launch_laswp_seq(double* a, long long lda, const int* blk, const int* ext, int base,
                     const int* widths, int lists, int c0, int c1, int c2, int c3,
                     cudaStream_t s);

// B(w x nc) <- L^{-1} B, L unit lower (w x w) at a(r0, r0), B at a(r0, c0);
// w <= trsm_max_width().  A non-null `gate`: do nothing when *gate >= 0
// (the stop word of an enqueued panel sequence, read when the kernel starts).
int trsm_max_width();
void launch_trsm_unit_lower(double* a, long long lda, int r0, int w, int c0, int nc,
                            cudaStream_t s, const int* gate = nullptr);
// T (w x w, column stride ldt) <- I - L^{-1} for the unit lower w x w block L,
// w <= lower_inverse_max_width(): the solve L^{-1} B is then B - T B, a GEMM.
int lower_inverse_max_width();
void launch_lower_inverse(const double* L, long long ldl, int w, double* T, long long ldt,
                          cudaStream_t s);
// dst <- src for a rows x cols column-major block (device memory).
void launch_copy_block(const double* src, long long lds, double* dst, long long ldd, int rows,
                       int cols, cudaStream_t s);
// Same with separate operands; and B <- U^{-1} B for upper U with diagonal.
void launch_trsm_lower_unit(const double* L, long long ldl, double* B, long long ldb, int w, int nc,
                            cudaStream_t s, const int* gate = nullptr);
void launch_trsm_upper(const double* U, long long ldu, double* B, long long ldb, int w, int nc,
                       cudaStream_t s);

// C(M x N) -= A(M x K) * B(K x N); all three inside the same column-major
// matrix (or any column-major operands).  `gate` as for the TRSM.
void launch_gemm_minus(int M, int N, int K, const double* A, long long lda, const double* B,
                       long long ldb, double* C, long long ldc, cudaStream_t s,
                       const int* gate = nullptr);

// Lower triangle of the symmetric N x N C -= A(N x K) * B(K x N); C's strict
// upper triangle is not written.
void launch_gemm_minus_lower(int N, int K, const double* A, long long lda, const double* B,
                             long long ldb, double* C, long long ldc, cudaStream_t s);

// C(M x N) -= A(M x K) * B(K x N) on the tensor cores (BF16 split into
// `terms` pieces: 2 -> three products, 3 -> six products; FP32 accumulation in
// TMEM); scratch of mixed_scratch_bytes(M, N, K, terms) bytes.  Returns a
// status code.
size_t mixed_scratch_bytes(int max_rows, int max_cols, int max_k, int terms);
int launch_gemm_minus_mixed(int M, int N, int K, const double* A, long long lda, const double* B,
                            long long ldb, double* C, long long ldc, void* scratch, int terms,
                            int* status, cudaStream_t s);
// Split pieces of a mixed precision (0 for DP_PRECISION_FP64).
inline int mixed_terms(int precision) {
  return precision == DP_PRECISION_MIXED_BF16X6 ? 3 : precision == DP_PRECISION_MIXED_BF16X3 ? 2 : 0;
}
inline bool valid_precision(int precision) {
  return precision == DP_PRECISION_FP64 || precision == DP_PRECISION_MIXED_BF16X3 ||
         precision == DP_PRECISION_MIXED_BF16X6;
}

// Full-pivot search over a(k:m, k:n); result in state->fallback.
void launch_search_active(const double* a, long long lda, int m, int n, int k, State* state,
                          Cand* block_cands, int max_blocks, cudaStream_t s);

// Column-fallback search (delayed_dgetrf_column.cpp:30-45): right-most column
// j in (k, n) whose active part has a magnitude > threshold, and its argmax row.
void launch_search_nonzero_column(const double* a, long long lda, int m, int n, int k,
                                  double threshold, State* state, cudaStream_t s);

// Swap full rows r1 <-> r2 over columns [0, n) and full columns c1 <-> c2 over
// rows [0, m) (either may be a no-op when the indices are equal).
void launch_swap_row(double* a, long long lda, int n, int r1, int r2, cudaStream_t s);
void launch_swap_col(double* a, long long lda, int m, int c1, int c2, cudaStream_t s);

void launch_identity_records(int* ipiv, int* jpiv, int count, cudaStream_t s);
void launch_set_record(int* ipiv, int* jpiv, int k, int p, int q, cudaStream_t s);

// ---- triangular solves with many right-hand sides (trisolve.cu) ----------

// Y (n x nrhs, nrhs <= tri_solve_rhs_max()) <- L^{-1} Y (unit lower) or
// U^{-1} Y (upper with diagonal), one launch; `flags` holds
// tri_solve_flag_count(n) words: one per 64-row block, whose values differ
// from `epoch` (nonzero, new for every launch that uses the same flags), then
// the launch's block-ticket counter (reset by the launch); a bounded wait
// that runs out sets *status = kDeviceTimeout.
// `inv` holds the inverses of the 64 x 64 diagonal blocks of L and U
// (launch_diag_inverse, tri_inverse_doubles(n) doubles, 16-byte aligned).
int tri_solve_rhs_max();
int tri_solve_flag_count(int n);
size_t tri_inverse_doubles(int n);
int launch_diag_inverse(const double* lu, long long ldlu, int n, double* inv, cudaStream_t st);
int launch_tri_lower_unit(const double* L, long long ldl, int n, const double* inv, double* Y,
                          long long ldy, int nrhs, unsigned* flags, unsigned epoch, int* status,
                          cudaStream_t st);
int launch_tri_upper(const double* U, long long ldu, int n, const double* inv, double* Y,
                     long long ldy, int nrhs, unsigned* flags, unsigned epoch, int* status,
                     cudaStream_t st);

// ---- resident factorisations (solve.cu) ----------------------------------

// A factorisation kept on the device for repeated solves: the compact L\U,
// its swap histories (host) and their composite row / column orders (device).
struct Factor {
  int n = 0;
  int info = -1;
  int precision = 0;                  // DP_PRECISION_* of the factors held now
  int refactored = 0;                 // 1 once a stalled refinement forced FP64
  double normA = 0.0;                 // ||A||_inf
  double factor_ms = 0.0;             // device time of all factorisations
  double* lu = nullptr;
  int* d_perm = nullptr;              // row order [n], column order [n]
  unsigned* d_flags = nullptr;        // triangular-solve block flags, then a status word
  double* d_inv = nullptr;            // inverses of the diagonal blocks of L and U
  unsigned epoch = 0;                 // last epoch used on d_flags
  int panel_rows = 0;                 // rows per panel CTA of its factorisations (0: default)
  std::vector<int> ipiv, jpiv;
};

// Device bytes a Factor of order n holds.
size_t factor_bytes(int n);
// Factor A (n x n, lda, device, not modified) at `precision`; synchronises st.
int factor_create(Factor** out, int n, const double* A, int lda, int precision, cudaStream_t st,
                  int panel_rows = 0);
// Solve A X = B with FP64 refinement; B (n x nrhs, device) becomes X.  Mixed
// factors whose refinement stalls are replaced by plain FP64 factors of A.
int factor_solve(Factor* f, const double* A, int lda, double* B, int ldb, int nrhs, int max_iter,
                 double tol, dp_ir_result* res, cudaStream_t st);
void factor_destroy(Factor* f, cudaStream_t st);
// Hager-Higham estimate of kappa_1(A) = ||A||_1 ||A^{-1}||_1 through the
// factors held now (inv_norm: the estimate of ||A^{-1}||_1, may be null);
// synchronises st.  A singular factorisation gives infinity.
int factor_condest(Factor* f, const double* A, int lda, double* kappa, double* inv_norm,
                   cudaStream_t st);

}  // namespace dp
