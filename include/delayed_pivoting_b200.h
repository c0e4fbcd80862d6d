/* C ABI of the B200 delayed-pivoting LU (libdelayed_lu_b200.so).
 *
 * Plain pointers and sizes only; `stream` is a cudaStream_t passed as void*
 * (NULL = the legacy default stream).  Return values are status codes:
 *   0 DP_SUCCESS, 1 DP_INVALID_ARGUMENT, 2 DP_ALLOCATION_FAILED,
 *   3 DP_CUDA_FAILURE, 4 DP_LIBRARY_FAILURE (the reference's cublas_failure),
 *   5 DP_DEVICE_TIMEOUT (a bounded device wait gave up).
 * The codes equal the reference's DelayedGetrfCudaStatus values
 * (delayed_lu_cuda/delayed_dgetrf_cuda.hpp:7-13) plus one.
 *
 * Matrix and record conventions are the reference's
 * (delayed_lu_cuda/delayed_dgetrf_cuda.hpp:15-26): column-major, 0-based,
 * in-place compact L\U, ipiv/jpiv are 0-based swap histories of min(m,n)
 * entries in HOST memory, info = min(m,n) or the first delayed step, -1 on
 * any failure.  Every entry point synchronises `stream` before returning.
 */
#ifndef DELAYED_PIVOTING_B200_H
#define DELAYED_PIVOTING_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DP_SUCCESS = 0,
  DP_INVALID_ARGUMENT = 1,
  DP_ALLOCATION_FAILED = 2,
  DP_CUDA_FAILURE = 3,
  DP_LIBRARY_FAILURE = 4,
  DP_DEVICE_TIMEOUT = 5
};

enum { DP_POLICY_FULL_PIVOT = 0, DP_POLICY_NONZERO_COLUMN = 1 };

/* Arithmetic of the O(n^3) trailing update.  Pivot search, delay / fallback
 * decisions, panel and TRSM are FP64 in every mode.  MIXED_BF16X3: BF16
 * hi/lo split, three tensor-core products (about 2^-16 relative per update);
 * MIXED_BF16X6: three-piece split, six products (about 2^-24, FP32-level),
 * both with FP32 accumulation. */
enum { DP_PRECISION_FP64 = 0, DP_PRECISION_MIXED_BF16X3 = 1, DP_PRECISION_MIXED_BF16X6 = 2 };

/* Tuning and semantics knobs; dp_options_init() fills the defaults that
 * reproduce the reference exactly (threshold 0, full-pivot fallback). */
typedef struct dp_options {
  int nb;            /* panel width (the reference fixes 64); 0 = automatic */
  double threshold;  /* accept a pivot iff |alpha| > threshold; 0 = reference */
  int policy;        /* DP_POLICY_FULL_PIVOT (delayed_getrf) or
                        DP_POLICY_NONZERO_COLUMN (delayed_getrf_column) */
  int panel_rows;    /* target rows per CTA in the panel kernel; 0 = automatic */
  int nb_outer;      /* outer block width of the trailing update; 0 = automatic */
  int panel_kernel;  /* 0 automatic (single-CTA panel up to 512 rows, else the cluster
                        panel), 1 cluster (sub-panel in registers up to 512 rows per
                        CTA), 2 grid-wide, 3 cluster with the sub-panel in shared memory */
  int precision;     /* DP_PRECISION_FP64 (reference arithmetic) or
                        DP_PRECISION_MIXED_BF16X3 (tensor-core trailing update) */
  int lookahead;     /* 0 automatic (on beyond one outer block), 1 on, 2 off: the
                        trailing update right of the next outer block runs on a
                        second stream behind the next block's panels */
} dp_options;

void dp_options_init(dp_options *opt);

/* Replaces delayed_getrf_cuda_device (delayed_lu_cuda/delayed_dgetrf_cuda.hpp:24-26,
 * delayed_dgetrf_cuda.cu:403-447).  d_a is device memory. */
int dp_getrf_device(int m, int n, double *d_a, int lda, int *ipiv, int *jpiv, int *info,
                    void *stream);

/* Replaces delayed_getrf_cuda_host (delayed_dgetrf_cuda.hpp:35-37,
 * delayed_dgetrf_cuda.cu:449-488).  a is host memory. */
int dp_getrf_host(int m, int n, double *a, int lda, int *ipiv, int *jpiv, int *info,
                  void *stream);

/* delayed_dgetrf_cuda.hpp:40-46 (native_*) and :55-61 (hybrid_*, which here
 * run the same all-device path). */
int dp_getrf_native_device(int m, int n, double *d_a, int lda, int *ipiv, int *jpiv, int *info,
                           void *stream);
int dp_getrf_native_host(int m, int n, double *a, int lda, int *ipiv, int *jpiv, int *info,
                         void *stream);
int dp_getrf_hybrid_device(int m, int n, double *d_a, int lda, int *ipiv, int *jpiv, int *info,
                           void *stream);
int dp_getrf_hybrid_host(int m, int n, double *a, int lda, int *ipiv, int *jpiv, int *info,
                         void *stream);

/* Allocation-free dp_getrf_device (no counterpart in the reference, which
 * allocates its temporaries with cudaMalloc on every call).  For callers that
 * cannot allocate device memory while factoring - a memory manager that owns
 * the whole pool, a fixed HBM budget, an allocator other than the CUDA
 * runtime's.  Same arguments, results and errors as dp_getrf_device (plain
 * FP64, reference semantics); its scratch is one 320 KiB array inside the
 * library, held on every GPU that loads the library until the process exits.
 * Limits: min(m,n) <= 32768 and the first panel must fit the cluster panel
 * kernel; larger inputs return DP_INVALID_ARGUMENT with info = -1.  All calls
 * share the array: calls that overlap on the GPU (other threads, other
 * streams) race and must be serialised by the caller.  The first call on a
 * device looks the array's device address up once (a host-side query that
 * allocates nothing).  Like every dp_getrf_* entry point it reads the pivot
 * state during the call and synchronises `stream` before returning. */
int dp_getrf_device_noalloc(int m, int n, double *d_a, int lda, int *ipiv, int *jpiv, int *info,
                            void *stream);

/* dp_getrf_device with explicit options (opt == NULL: defaults).  Also the
 * column-fallback policy of delayed_lu/delayed_dgetrf_column.hpp:18. */
int dp_getrf_device_ex(int m, int n, double *d_a, int lda, int *ipiv, int *jpiv, int *info,
                       void *stream, const dp_options *opt);

/* Panel-width autotuner of the single-matrix LU (no reference counterpart:
 * the reference fixes block_size = 64, delayed_lu/delayed_dgetrf.cpp:16).
 * Times the (panel width nb, outer block nb_outer) pairs {32, 64, 128} x
 * {64, 128, 256} (nb <= nb_outer) on a seeded N(0,1) n x n matrix, best of
 * two runs each, and records the fastest pair for n's order bucket
 * [2^b, 2^(b+1)) on the current device.  Every dp_getrf_* call whose caller
 * leaves both widths automatic (no options, or nb = nb_outer = 0) then uses
 * the pair of its min(m, n) bucket.  Widths change rounding only, never the
 * records.  Allocates 2 n^2 doubles while it runs; synchronises `stream`.
 * dp_getrf_tune_save / _load write / read the current device's table
 * ("<smallest n> <largest n> <nb> <nb_outer>" per tuned bucket). */
int dp_getrf_autotune(int n, int *nb, int *nb_outer, void *stream);
int dp_getrf_tune_save(const char *path);
int dp_getrf_tune_load(const char *path);

/* Near-tie report (no reference counterpart; the reference decides every
 * pivot by a bare argmax, delayed_lu/delayed_dgetrf.cpp:170-178 and :32-47,
 * delayed_lu_cuda/delayed_dgetrf_cuda.cu:13-20).  Every pivot decision of a
 * factorisation - the column search of each panel step and each fallback
 * search - also finds the runner-up magnitude.  A decision is order-sensitive
 * when (best - second) <= 4 (k + 1) u best (u = 2^-53, k the step): the
 * rounding of another summation order could swap the two, so a records match
 * with the reference is only meaningful where near_ties == 0.  Decisions on a
 * zero winner (stop / delay) are exact and never count.  Not covered: the
 * grid-wide panel kernel (dp_options.panel_kernel = 2, or panels too tall for
 * a 16-CTA cluster), whose steps are not counted in `decisions`. */
typedef struct dp_getrf_report {
  long long decisions;  /* pivot decisions whose runner-up was compared */
  long long near_ties;  /* order-sensitive decisions among them */
  double max_closeness; /* largest second / best over those decisions (1: an exact tie) */
  int info;             /* info of the call (-1: the call failed) */
  int reserved[3];
} dp_getrf_report;

/* The report of the calling host thread's last dp_getrf_* call (device, host,
 * _ex, _noalloc; C++ delayed_getrf_cuda_* alike). */
int dp_getrf_last_report(dp_getrf_report *report);

/* Solve A X = B with the factors of dp_getrf_device (no reference
 * counterpart: the reference stops at the factorisation).  P*A*Q = L*U from
 * the swap histories ipiv / jpiv (HOST arrays of n entries, as returned by
 * dp_getrf_*); the factorisation must be complete (info == n).  d_b (n x nrhs,
 * device) is overwritten with X.  Synchronises `stream`. */
int dp_getrs_device(int n, int nrhs, const double *d_lu, int ldlu, const int *ipiv,
                    const int *jpiv, double *d_b, int ldb, void *stream);

typedef struct dp_ir_result {
  int info;              /* factorisation info of the last factorisation */
  int iterations;        /* refinement corrections applied (all factorisations) */
  int refactored;        /* 1 when the mixed factors stalled and FP64 was used */
  int converged;         /* 1 when backward_error <= tol */
  double backward_error; /* max_c ||b_c - A x_c||_inf / (||A||_inf ||x_c||_inf + ||b_c||_inf) */
  double factor_ms;      /* device time of the factorisation(s) */
  double total_ms;       /* device time of the whole solve */
} dp_ir_result;

/* Solve A X = B by a (mixed-precision) delayed LU and FP64 iterative
 * refinement (no reference counterpart).  d_a (n x n) is not modified; d_b
 * (n x nrhs) is overwritten with X.  precision: DP_PRECISION_*; refinement
 * stops at backward error <= tol, after max_iter corrections, or when the
 * error stops halving - then a mixed-precision solve is re-factored in FP64.
 * Synchronises `stream`. */
int dp_gesv_ir_device(int n, int nrhs, const double *d_a, int lda, double *d_b, int ldb,
                      int precision, int max_iter, double tol, dp_ir_result *result,
                      void *stream);

/* ---- Resident factorisations (no reference counterpart): factor once, solve
 * many right-hand sides later with FP64 refinement.  The factors live on the
 * device until dp_factor_destroy; the caller keeps d_a (the matrix the
 * factors came from, needed for the refinement residuals) valid and
 * unmodified meanwhile. */
typedef struct dp_factor dp_factor;
/* Factor d_a (n x n, device, not modified) at `precision` (DP_PRECISION_*).
 * Synchronises `stream`.  A singular matrix gives a factor with info < n.
 * Mixed-precision factors whose pivot range max |u_ii| / min |u_ii| exceeds
 * 1e8 (a lower bound on kappa(U) at which refinement from ~2^-24 factors
 * would stall) are replaced by plain FP64 factors at once (dp_ir_result
 * .refactored = 1 on its solves). */
int dp_factor_create(dp_factor **factor, int n, const double *d_a, int lda, int precision,
                     void *stream);
/* info of the factorisation, precision of the factors held now (a stalled
 * mixed-precision refinement replaces them by FP64 factors), device
 * milliseconds of all factorisations so far; outputs may be NULL. */
int dp_factor_info(const dp_factor *factor, int *info, int *precision, double *factor_ms);
/* Solve A X = B: d_b (n x nrhs, device) becomes X; refinement as in
 * dp_gesv_ir_device.  Synchronises `stream`. */
int dp_factor_solve(dp_factor *factor, const double *d_a, int lda, double *d_b, int ldb,
                    int nrhs, int max_iter, double tol, dp_ir_result *result, void *stream);
/* Condition estimate (no reference counterpart): Hager's 1-norm estimator
 * with Higham's safeguards (LAPACK dlacon's algorithm: at most 5 iterations,
 * then the alternating-sign vector), i.e. kappa_1(A) ~= ||A||_1 ||A^{-1}||_1
 * from a handful of solves with A and A^T through the resident factors -
 * usually within a factor 3 of the true value, never above it.  d_a is the
 * matrix the factors came from; mixed-precision factors estimate the
 * condition of the matrix they factor exactly.  A singular factorisation
 * (info < n) gives infinity.  Allocates n*n doubles of scratch for the
 * duration of the call; synchronises `stream`. */
int dp_factor_condest(dp_factor *factor, const double *d_a, int lda, double *kappa1,
                      void *stream);
void dp_factor_destroy(dp_factor *factor, void *stream);

/* ---- Batched factorisation (no reference counterpart: the reference factors
 * one matrix per call).  Thousands of independent square matrices of orders
 * 1..DP_BATCH_MAX_N, each column-major with lda = its order, factored by ONE
 * persistent kernel launch that pulls matrices from a device work queue
 * (largest first).  Each matrix gets exactly the single-matrix semantics of
 * dp_getrf_device (delayed_lu/delayed_dgetrf.cpp:129-251): same records, same
 * info, compact L\U in place.  Records stay on the device: matrix i's ipiv /
 * jpiv are the n_i entries at its record offset, info[i] its info. */
#define DP_BATCH_MAX_N 512
#define DP_BATCH_MAX_NB 32
#define DP_BATCH_BUCKETS 4 /* panel-width buckets: n < 64, < 128, < 256, <= 512 */

typedef struct dp_batch_options {
  double threshold;                /* accept a pivot iff |alpha| > threshold */
  int precision;                   /* DP_PRECISION_FP64 (the single-matrix semantics and
                                      records), or DP_PRECISION_MIXED_BF16X3 / _BF16X6: the
                                      trailing updates A22 -= L21 U12 as BF16 split
                                      products (3 / 6, FP32 accumulation, on mma.sync
                                      m16n8k16), panels, U12 solves, searches and pivot
                                      decisions in FP64; factors for FP64 refinement,
                                      records may differ where a decision is within the
                                      update's rounding */
  int nb_bucket[DP_BATCH_BUCKETS]; /* panel width per order bucket, 1..DP_BATCH_MAX_NB */
  int reserved[2];
} dp_batch_options;

void dp_batch_options_init(dp_batch_options *opt);

typedef struct dp_batch dp_batch; /* a plan: the orders, the layout, the queue */

/* n: host array of `count` orders.  offsets: host array of each matrix's
 * first element in the caller's buffer, or NULL for the packed layout (each
 * matrix after the previous one, rounded up to 4 elements).  Allocates the
 * plan's small device arrays (on the current device). */
int dp_batch_create(dp_batch **plan, int count, const int *n, const long long *offsets,
                    const dp_batch_options *opt);
/* The plan's matrix offsets (elements), record offsets, buffer and record
 * totals; any output may be NULL. */
int dp_batch_layout(const dp_batch *plan, long long *offsets, long long *record_offsets,
                    long long *total_elements, long long *total_records);
int dp_batch_set_options(dp_batch *plan, const dp_batch_options *opt);
/* Enqueue the factorisation of every matrix of d_base on `stream` (device
 * records d_ipiv / d_jpiv of total_records entries, d_info of count); returns
 * without synchronising and may be captured into a CUDA graph.  One plan runs
 * one launch at a time (the launches share the plan's work counter). */
int dp_batch_getrf_async(dp_batch *plan, double *d_base, int *d_ipiv, int *d_jpiv, int *d_info,
                         void *stream);
/* The same launch replayed from a CUDA graph the plan captures on first use
 * (and again when the pointers or options change). */
int dp_batch_getrf_graph(dp_batch *plan, double *d_base, int *d_ipiv, int *d_jpiv, int *d_info,
                         void *stream);
void dp_batch_destroy(dp_batch *plan);
/* Near-tie report (see dp_getrf_report) summed over every matrix of the
 * plan's last launch; `info` holds the number of matrices.  Synchronises the
 * device (cudaDeviceSynchronize) before it reads the plan's counters. */
int dp_batch_last_report(dp_batch *plan, dp_getrf_report *report);

/* Autotuner: for each bucket, times every candidate panel width on `samples`
 * seeded N(0,1) matrices whose orders spread log-uniformly over the bucket,
 * and writes the fastest into opt->nb_bucket.  Synchronises `stream`. */
int dp_batch_autotune(dp_batch_options *opt, int samples, unsigned long long seed, void *stream);
/* Tuning table file: one line per bucket, "<smallest n> <largest n> <nb>". */
int dp_batch_tune_save(const char *path, const dp_batch_options *opt);
int dp_batch_tune_load(const char *path, dp_batch_options *opt);

/* ---- Serving (no reference counterpart): a request loop on one GPU.
 * Requests to factor a matrix and solve right-hand sides arrive at any time
 * from any host thread; the server admits them against an HBM budget as
 * memory frees up, sends orders <= small_max_n through the persistent batched
 * factorisation (many requests per launch) and larger ones through the
 * blocked factorisation on concurrent streams, refines every solve in FP64,
 * and keeps factors resident for follow-up solves.  Every solve of a request
 * is computed the same way whether it runs alone or among others.
 * The server works on its own streams: a request's device buffers must hold
 * their data when it is submitted (synchronise the stream that wrote them),
 * and X is in d_b once the request's result has been polled. */
typedef struct dp_server_options {
  unsigned long long budget_bytes; /* HBM admission budget (0: 160 GB) */
  int precision;       /* DP_PRECISION_* of the blocked factorisations (default: MIXED_BF16X6) */
  int large_workers;   /* concurrent blocked factorisations (streams); 0: 6 */
  int small_max_n;     /* orders up to this take the batched path (<= DP_BATCH_MAX_N); 0: 512,
                          -1: none */
  int small_max_batch; /* requests per batched launch; 0: 2048 */
  int max_iter;        /* refinement steps per solve; 0: 10 */
  double tol;          /* backward-error target; 0: 1e-14 */
  int panel_rows;      /* rows per CTA of the large factorisations' cluster panels (fewer CTAs
                          per panel: less SM time, more latency); 0: the library default (256) */
  int mixed_min_n;     /* with a mixed `precision`, blocked factorisations of a lower order use
                          FP64 factors: measured on B200, the BF16-split update and its
                          refinement cost more than the FP64 factorisation below n ~ 12,000
                          (factor + refined solve, kappa <= 1e4: 8192 -> 39.6 against 38.4 ms,
                          12288 -> 69 against 81 ms); 0: 12288, -1: every order mixed */
  int reserved[2];
} dp_server_options;

void dp_server_options_init(dp_server_options *opt);

typedef struct dp_request {
  unsigned long long id;        /* caller's tag, unique among live requests, != 0 */
  unsigned long long factor_id; /* 0: factor d_a; else a follow-up solve on the resident
                                   factors of request factor_id */
  int n;
  const double *d_a;            /* n x n, device; read only; must stay valid until the
                                   request's factors are released */
  int lda;
  double *d_b;                  /* n x nrhs right-hand sides, device; becomes X */
  int ldb;
  int nrhs;                     /* 1..64 */
  int followups;                /* new factorisation: number of follow-up solves that will
                                   name it; its factors stay resident until they are done */
  int reserved;
} dp_request;

typedef struct dp_request_result {
  unsigned long long id;
  int status;            /* DP_* */
  int info;              /* factorisation info (n: nonsingular) */
  int precision;         /* arithmetic of the factors that produced X */
  int iterations;        /* refinement corrections */
  int refactored;        /* 1: mixed factors stalled, re-factored in FP64 */
  int path;              /* 0: batched (small), 1: blocked (large) */
  double backward_error; /* max_c ||b_c - A x_c||_inf / (||A||_inf ||x_c||_inf + ||b_c||_inf) */
  double t_submit, t_admit, t_start, t_done; /* dp_server_clock() seconds */
  double factor_ms;      /* large path: device time of the factorisation(s) on the worker's
                            stream (events; includes waits for SMs held by other requests) */
  double solve_ms;       /* large path: device time of the solve and its refinement */
} dp_request_result;

typedef struct dp_server_stats {
  unsigned long long bytes_in_use, bytes_peak;
  long long submitted, completed, pending, residents;
  long long small_launches, small_items, large_items;
} dp_server_stats;

typedef struct dp_server dp_server;
/* Creates the server on the current device and starts its host threads. */
int dp_server_create(dp_server **server, const dp_server_options *opt);
/* Queues a request (thread-safe, returns at once).  DP_INVALID_ARGUMENT for
 * bad sizes or pointers, a duplicate id, or a request that can never fit the
 * budget. */
int dp_server_submit(dp_server *server, const dp_request *request);
/* Moves up to `max` completed results into `out`, waiting up to wait_ms for
 * the first one; returns how many were moved. */
int dp_server_poll(dp_server *server, dp_request_result *out, int max, int wait_ms);
int dp_server_stats_get(dp_server *server, dp_server_stats *out);
/* Seconds on the server's monotonic clock (the timestamps of the results). */
double dp_server_clock(void);
/* Waits for every queued request, releases all resident factors, stops. */
void dp_server_destroy(dp_server *server);

/* Per-kernel-family device timing (no reference counterpart; the reference
 * only times whole calls with std::chrono, delayed_lu_cuda/benchmark.cu:54-57).
 * When enabled, every call records CUDA events around each launch group on
 * its stream and accumulates device milliseconds, launches and algorithmic
 * flops / bytes per family. */
enum {
  DP_KFAM_PANEL = 0, /* panel factorisation (search, swap, scale, rank-1) */
  DP_KFAM_LASWP = 1, /* row permutation of the columns outside the panel */
  DP_KFAM_TRSM = 2,  /* U12 = L11^-1 A12 */
  DP_KFAM_GEMM = 3,  /* A22 -= L21 U12 (FP64 DMMA) */
  DP_KFAM_SEARCH = 4,/* fallback search over the active submatrix */
  DP_KFAM_SWAP = 5,  /* fallback full-row / full-column swaps and records */
  DP_KFAM_OTHER = 6, /* record initialisation */
  DP_KFAM_GEMM_MIXED = 7, /* A22 -= L21 U12 on tcgen05 (BF16x3, incl. operand split) */
  DP_KFAM_COUNT = 8
};
typedef struct dp_kernel_stats {
  double ms[8];
  double flops[8];
  double bytes[8];
  long long launches[8];
  long long calls;
} dp_kernel_stats;
void dp_stats_enable(int on);
/* Families recorded while enabled: bit DP_KFAM_x set (default all, ~0u);
 * fewer families mean fewer timing events inside the timed work.  Returns
 * the previous mask. */
unsigned dp_stats_families(unsigned mask);
void dp_stats_reset(void);
void dp_stats_get(dp_kernel_stats *out);

/* Kernel launches this library has issued since it was loaded, on every
 * stream and host thread (no reference counterpart). */
long long dp_kernel_launches(void);

/* The FP64 Schur-complement update of the factorisation, C -= A * B, on the
 * DMMA tensor-core kernel (column-major M x K A, K x N B, M x N C; the
 * trailing update that delayed_dgetrf_cuda.cu:205-209 hands to cublasDgemm
 * with alpha = -1, beta = 1).  Asynchronous on `stream`; every element is
 * accumulated over k in order, one FP64 accumulator. */
int dp_schur_update_device(int M, int N, int K, const double *A, int lda, const double *B,
                           int ldb, double *C, int ldc, void *stream);

/* The same update on the tensor cores, as the mixed-precision factorisation
 * runs it (precision DP_PRECISION_MIXED_BF16X3 / _BF16X6: A and B split into
 * 2 / 3 BF16 pieces, 3 / 6 products, FP32 accumulation in tensor memory, C -=
 * acc in FP64).  Scratch for the pieces comes from the stream-ordered pool;
 * synchronises `stream`.  Returns DP_DEVICE_TIMEOUT if a bounded wait of the
 * kernel gave up. */
int dp_schur_update_mixed_device(int M, int N, int K, const double *A, int lda, const double *B,
                                 int ldb, double *C, int ldc, int precision, void *stream);

/* Tile of that kernel for N > 32 (tuning; no result bit depends on it):
 * 0 automatic (= 5), 1 128 x 128 (one CTA per SM), 2 128 x 64 (two CTAs per
 * SM), 3 64 x 64 (three CTAs per SM), 4 128 x 64 with eight warps, 5 64 x 64
 * with two stages (four CTAs per SM), 6 64 x 128 with four warps, 7 64 x 128
 * with eight warps, 8 64 x 64 with 32-deep k chunks.
 * Returns the previous setting, or -1 for an invalid one. */
int dp_gemm_tile(int tile);

/* CTAs of one triangular-solve launch of the solve / refinement path (tuning;
 * no result bit depends on it): 0 automatic (min(row blocks, SMs)), g > 0 at
 * most g, g < 0 one CTA per -g blocks of 64 rows (at most 32).  Returns the
 * previous setting, or -2000 for a setting outside [-1024, 1024]. */
int dp_tri_solve_grid(int policy);

/* CTAs of the tensor-core (mixed) update (tuning; no result bit depends on
 * it): 0 automatic (one per tile), g > 0 at most g, -1 one per SM (persistent
 * over the tiles).  Returns the previous setting, or -2 for an invalid one. */
int dp_mixed_gemm_grid(int policy);

/* How the factorisations solve the triangular systems of their outer blocks
 * (U12 = L11^{-1} A12 for blocks wider than 64 rows): 0 automatic (= 1),
 * 1 by inverse (T = I - L11^{-1} once per block, then U12 = A12 - T A12 on
 * the FP64 tensor path), 2 by substitution (64-row solves chained with
 * updates).  Process-wide; the two differ in rounding only (pivot records
 * differ only where a decision is a near tie).  The allocation-free entry
 * point always uses substitution.  Returns the previous setting, or -1 for an
 * invalid one. */
int dp_block_solve(int mode);

/* ---- Multifrontal hand-off (no reference code; the reference's design
 * document, doc/...LU方法.md:228-457).  A frontal matrix F (m x n, device,
 * column-major, ldf) whose leading p rows and p columns are fully summed is
 * factored partially: pivots are chosen inside the fully-summed block only,
 * with the delayed-pivoting rules of dp_getrf_device on F(0:p, 0:p) (records
 * ipiv / jpiv: host arrays of p entries, relative to the block; *npiv = k,
 * its info); the k eliminated pivots' L and U are applied to the whole front,
 * and F(k:m, k:n) becomes the contribution block for the parent front: the
 * Schur complement of the k pivots, its first p - k rows and columns the
 * delayed ones.  row_index / col_index (host, m and n entries, may be NULL):
 * the front's global row and column indices; their first p entries are
 * permuted into the factor's order, so row_index[k:m] and col_index[k:n]
 * index the contribution block.  0 <= p <= min(m, n).  Synchronises
 * `stream`. */
int dp_front_factor(int m, int n, int p, double *d_f, int ldf, int *row_index, int *col_index,
                    int *ipiv, int *jpiv, int *npiv, void *stream);
/* Extend-add of a child's contribution block into its parent front:
 * P(prow[i], pcol[j]) += C(i, j) for C (mc x nc, device, ldc); prow / pcol
 * (device, mc and nc entries) are the positions in the parent of the child's
 * rows and columns (distinct within one call).  Enqueued on `stream`, does
 * not synchronise; contributions of several children are ordered by the
 * stream. */
int dp_extend_add(int mc, int nc, const double *d_c, int ldc, const int *d_prow,
                  const int *d_pcol, double *d_p, int ldp, void *stream);

/* ---- Delayed Bunch-Kaufman LDL^T (delayed-bunch-kaufman/delayed_sytrf*.hpp) ----
 * Symmetric indefinite A (column-major, lda >= n, LOWER triangle read and
 * written, the strict upper triangle untouched) is factored in place as
 * P A P^T = L D L^T with Bunch-Kaufman 1x1 / 2x2 pivots (alpha =
 * (1 + sqrt 17) / 8), nodes whose pivots fail every test delayed to the end:
 *   perm[pos]     original index at position pos (host, n entries);
 *   piv_size[pos] 1 (1x1 pivot), 2 (first column of a 2x2 block), 0 (second
 *                 column of a 2x2 block, or delayed) (host, n entries);
 *   info          start of the delayed suffix (n when nothing is delayed),
 *                 -1 on failure;
 *   L's multipliers below the diagonal (a 2x2 block's start at k + 2), D on
 *   the diagonal with a 2x2 block's off-diagonal at (k + 1, k), and the
 *   delayed suffix's trailing block holding its Schur complement.
 * The records equal the reference's delayed_sytrf_blocked
 * (delayed_sytrf_blocked.cpp:141) and delayed_sytrf (delayed_sytrf.cpp:175)
 * wherever no decision is order-sensitive (dp_sytrf_last_report).  NaN never
 * wins the column search. */
typedef struct dp_sytrf_options {
  int nb;    /* panel width, 2..64 (the reference fixes 64); 0 = 64 */
  int grid;  /* CTAs of the panel kernel; 0 = one per 128 rows, at most one per SM.
                n may not exceed 512 rows per CTA (75776 with one CTA per SM). */
  int reserved[6];
} dp_sytrf_options;

void dp_sytrf_options_init(dp_sytrf_options *opt);
/* d_a device memory; synchronises `stream`. */
int dp_sytrf_device(int n, double *d_a, int lda, int *perm, int *piv_size, int *info,
                    void *stream);
int dp_sytrf_device_ex(int n, double *d_a, int lda, int *perm, int *piv_size, int *info,
                       const dp_sytrf_options *opt, void *stream);
/* a host memory (copied to the current GPU and back). */
int dp_sytrf_host(int n, double *a, int lda, int *perm, int *piv_size, int *info);
/* Near-tie report of the calling thread's last dp_sytrf_* call: decisions
 * counted, and how many had a comparison (column search runner-up, the three
 * Bunch-Kaufman tests, the 2x2 determinant test) within a relative
 * 4 (k + 1) u of flipping. */
int dp_sytrf_last_report(dp_getrf_report *report);

/* delayed_dgetrf_cuda.hpp:63 (delayed_getrf_cuda_status_string). */
const char *dp_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif
