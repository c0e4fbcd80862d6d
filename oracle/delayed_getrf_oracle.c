/*
 * CPU restatement of the reference's blocked delayed-pivoting LU.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA library is
 * checked against; it is imported by tests/, by __graft_entry__.smoke() and by
 * the CPU leg of bench.py, and by nothing in the product library.
 *
 * It restates, step by step and with plain loops instead of BLAS calls,
 *   delayed_lu/delayed_dgetrf.cpp:129-251         (delayed_getrf)
 *   delayed_lu/delayed_dgetrf_column.cpp:99-211   (delayed_getrf_column)
 * with two parameters the reference fixes at compile time or leaves out:
 *   nb        panel width (delayed_dgetrf.cpp:16 fixes 64).  Panel width only
 *             changes rounding, never the pivot decisions.
 *   threshold absolute acceptance threshold; a pivot candidate is accepted iff
 *             |alpha| > threshold.  threshold = 0 is exactly the reference's
 *             `!(alpha > 0.0)` test (delayed_dgetrf.cpp:178, :189).
 * Pivot search semantics follow the reference's GPU twin
 * (delayed_lu_cuda/delayed_dgetrf_cuda.cu:13-20, :46): larger magnitude wins,
 * ties go to the earlier element in column-major order, NaN never wins.
 *
 * Records: ipiv[k] / jpiv[k] are the 0-based row / column swapped with k at
 * step k (a swap history, delayed_dgetrf.cpp:198-209); entries >= info stay
 * identity.  info = min(m,n) when nothing is delayed, k when the whole active
 * submatrix from step k on has no acceptable pivot, -1 for invalid arguments.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX(r, c, ld) ((size_t)(r) + (size_t)(c) * (size_t)(ld))

/* argmax |x[0..len)|, first index on ties, NaN never wins (initial best is
 * element 0 with magnitude 0 unless element 0 is a number). */
static int col_argmax(int len, const double *x, double *best_abs) {
  int best = 0;
  double b = 0.0;
  for (int i = 0; i < len; ++i) {
    double v = fabs(x[i]);
    if (v > b) {
      b = v;
      best = i;
    }
  }
  *best_abs = b;
  return best;
}

/* delayed_dgetrf.cpp:32-47: argmax over A(k:m, k:n), column-major order
 * tie-break (smaller column, then smaller row). */
static void find_active_max(int m, int n, const double *a, int lda, int k,
                            int *row, int *col, double *val) {
  int br = k, bc = k;
  double bv = 0.0;
  for (int j = k; j < n; ++j) {
    double v;
    int r = k + col_argmax(m - k, a + IDX(k, j, lda), &v);
    if (v > bv) {
      bv = v;
      br = r;
      bc = j;
    }
  }
  *row = br;
  *col = bc;
  *val = bv;
}

/* delayed_dgetrf_column.cpp:30-45: right-to-left first column whose active
 * part holds an acceptable entry; its column argmax row. */
static void find_nonzero_column(int m, int n, const double *a, int lda, int k,
                                double threshold, int *row, int *col,
                                double *val) {
  for (int j = n - 1; j > k; --j) {
    double v;
    int r = k + col_argmax(m - k, a + IDX(k, j, lda), &v);
    if (v > threshold) {
      *row = r;
      *col = j;
      *val = v;
      return;
    }
  }
  *row = k;
  *col = k;
  *val = 0.0;
}

static void swap_rows(int n, double *a, int lda, int r1, int r2) {
  for (int j = 0; j < n; ++j) {
    double t = a[IDX(r1, j, lda)];
    a[IDX(r1, j, lda)] = a[IDX(r2, j, lda)];
    a[IDX(r2, j, lda)] = t;
  }
}

static void swap_cols(int m, double *a, int lda, int c1, int c2) {
  double *x = a + IDX(0, c1, lda), *y = a + IDX(0, c2, lda);
  for (int i = 0; i < m; ++i) {
    double t = x[i];
    x[i] = y[i];
    y[i] = t;
  }
}

/* B(w x nc) <- L^{-1} B with L unit lower (w x w), both column-major. */
static void trsm_unit_lower(int w, int nc, const double *l, int ldl, double *b,
                            int ldb) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nc; ++j) {
    double *bj = b + IDX(0, j, ldb);
    for (int p = 0; p < w; ++p) {
      const double u = bj[p];
      if (u == 0.0) continue;
      const double *lp = l + IDX(0, p, ldl);
      for (int i = p + 1; i < w; ++i) bj[i] -= lp[i] * u;
    }
  }
}

/* C(M x N) -= A(M x K) * B(K x N), column-major. */
static void gemm_minus(int M, int N, int K, const double *a, int lda,
                       const double *b, int ldb, double *c, int ldc) {
  if (M <= 0 || N <= 0 || K <= 0) return;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < N; ++j) {
    double *cj = c + IDX(0, j, ldc);
    const double *bj = b + IDX(0, j, ldb);
    for (int p = 0; p < K; ++p) {
      const double u = bj[p];
      if (u == 0.0) continue;
      const double *ap = a + IDX(0, p, lda);
      for (int i = 0; i < M; ++i) cj[i] -= ap[i] * u;
    }
  }
}

/* delayed_dgetrf.cpp:61-85 */
static void finish_panel(int m, int n, double *a, int lda, int begin, int end) {
  const int width = end - begin, cols_right = n - end;
  if (width <= 0 || cols_right <= 0) return;
  trsm_unit_lower(width, cols_right, a + IDX(begin, begin, lda), lda,
                  a + IDX(begin, end, lda), lda);
  gemm_minus(m - end, cols_right, width, a + IDX(end, begin, lda), lda,
             a + IDX(begin, end, lda), lda, a + IDX(end, end, lda), lda);
}

/* delayed_dgetrf.cpp:101-125 */
static void materialize_partial_panel(int m, int n, double *a, int lda,
                                      int begin, int k, int panel_end) {
  const int width = k - begin, far_cols = n - panel_end;
  if (width <= 0 || far_cols <= 0) return;
  trsm_unit_lower(width, far_cols, a + IDX(begin, begin, lda), lda,
                  a + IDX(begin, panel_end, lda), lda);
  gemm_minus(m - k, far_cols, width, a + IDX(k, begin, lda), lda,
             a + IDX(begin, panel_end, lda), lda, a + IDX(k, panel_end, lda),
             lda);
}

/* policy 0: full-pivot fallback (delayed_getrf); 1: nonzero-column fallback
 * (delayed_getrf_column). */
int oracle_delayed_getrf(int m, int n, double *a, int lda, int *ipiv,
                         int *jpiv, int *info, int nb, double threshold,
                         int policy) {
  *info = -1;
  if (m < 0 || n < 0 || lda < (m > 1 ? m : 1) || nb < 1 || !(threshold >= 0.0))
    return -1;
  const int pivots = m < n ? m : n;
  if ((m > 0 && n > 0 && a == NULL) ||
      (pivots > 0 && (ipiv == NULL || jpiv == NULL)))
    return -1;
  *info = pivots;
  for (int j = 0; j < pivots; ++j) ipiv[j] = jpiv[j] = j;

  int panel_begin = 0, positioned = 0;
  while (panel_begin < pivots) {
    const int panel_end = pivots < panel_begin + nb ? pivots : panel_begin + nb;
    int restart = 0;
    for (int k = panel_begin; k < panel_end; ++k) {
      if (positioned) {
        positioned = 0;
      } else {
        double alpha;
        int prow = k + col_argmax(m - k, a + IDX(k, k, lda), &alpha);
        int pcol = k;
        const int fallback = !(alpha > threshold);
        if (fallback) {
          if (k > panel_begin)
            materialize_partial_panel(m, n, a, lda, panel_begin, k, panel_end);
          int gr, gc;
          double gv;
          if (policy == 0)
            find_active_max(m, n, a, lda, k, &gr, &gc, &gv);
          else
            find_nonzero_column(m, n, a, lda, k, threshold, &gr, &gc, &gv);
          if (!(gv > threshold)) {
            *info = k;
            return 0;
          }
          prow = gr;
          pcol = gc;
        }
        ipiv[k] = prow;
        jpiv[k] = pcol;
        if (prow != k) swap_rows(n, a, lda, k, prow);
        if (pcol != k) swap_cols(m, a, lda, k, pcol);
        if (fallback && k > panel_begin) {
          panel_begin = k;
          positioned = 1;
          restart = 1;
          break;
        }
      }
      const int rows_below = m - k - 1;
      if (rows_below > 0) {
        const double inv = 1.0 / a[IDX(k, k, lda)];
        double *lk = a + IDX(k + 1, k, lda);
        for (int i = 0; i < rows_below; ++i) lk[i] *= inv;
      }
      const int pcr = panel_end - k - 1;
      if (rows_below > 0 && pcr > 0) {
        const double *lk = a + IDX(k + 1, k, lda);
        for (int j = k + 1; j < panel_end; ++j) {
          const double u = a[IDX(k, j, lda)];
          double *cj = a + IDX(k + 1, j, lda);
          for (int i = 0; i < rows_below; ++i) cj[i] -= lk[i] * u;
        }
      }
    }
    if (restart) continue;
    finish_panel(m, n, a, lda, panel_begin, panel_end);
    panel_begin = panel_end;
  }
  return 0;
}

/* Replay of a swap history into permutation vectors (example.cu:61-68):
 * row_order[i] = original row that ends up at row i, same for columns.  Only
 * the first `steps` records are replayed. */
void oracle_swap_history_to_perm(int m, int n, int steps, const int *ipiv,
                                 const int *jpiv, int *row_order,
                                 int *col_order) {
  for (int i = 0; i < m; ++i) row_order[i] = i;
  for (int j = 0; j < n; ++j) col_order[j] = j;
  for (int k = 0; k < steps; ++k) {
    int t = row_order[k];
    row_order[k] = row_order[ipiv[k]];
    row_order[ipiv[k]] = t;
    t = col_order[k];
    col_order[k] = col_order[jpiv[k]];
    col_order[jpiv[k]] = t;
  }
}

/* ||P A Q - Lbar Ubar||_F and ||A||_F for the compact storage the reference
 * produces (delayed_lu_cuda/example.cu:24-80): columns < info hold unit-lower
 * L, rows < info hold U from the diagonal on, and the block
 * [info:m, info:n] holds the remaining Schur complement (an identity block of
 * Lbar times those rows of Ubar).  out[0] = residual, out[1] = ||A||_F.
 * `work` holds m doubles per OpenMP thread (m * omp_get_max_threads()). */
void oracle_residual(int m, int n, const double *orig, int lda_o,
                     const double *fac, int lda_f, int info, const int *ipiv,
                     const int *jpiv, double *out, int *row_order,
                     int *col_order, double *work) {
  oracle_swap_history_to_perm(m, n, info, ipiv, jpiv, row_order, col_order);
  double res = 0.0, an = 0.0;
#pragma omp parallel reduction(+ : res, an)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double *t = work + (size_t)tid * (size_t)m;
#pragma omp for schedule(dynamic, 8)
    for (int j = 0; j < n; ++j) {
      for (int i = 0; i < m; ++i) t[i] = 0.0;
      const int pmax = info < j + 1 ? info : j + 1;
      for (int p = 0; p < pmax; ++p) {
        const double u = fac[IDX(p, j, lda_f)];
        if (u == 0.0) continue;
        const double *lp = fac + IDX(0, p, lda_f);
        for (int i = p + 1; i < m; ++i) t[i] += lp[i] * u;
      }
      for (int i = 0; i < m; ++i) {
        if (i < info ? j >= i : j >= info) t[i] += fac[IDX(i, j, lda_f)];
        const double e = orig[IDX(row_order[i], col_order[j], lda_o)];
        const double d = t[i] - e;
        res += d * d;
        an += e * e;
      }
    }
  }
  out[0] = sqrt(res);
  out[1] = sqrt(an);
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
