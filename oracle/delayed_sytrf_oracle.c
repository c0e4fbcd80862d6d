/* Plain-C restatement of the reference's blocked delayed Bunch-Kaufman LDL^T
 * (delayed-bunch-kaufman/delayed_sytrf_blocked.cpp), used as a CHECKER only:
 * tests/ and bench.py's CPU arm call it; the product library never links it.
 *
 * Pinned against the reference's own records: tests/test_sytrf.py compares
 * perm / piv_size / info of this restatement with fixtures generated by the
 * reference's compiled delayed_sytrf_blocked and delayed_sytrf
 * (tests/golden/make_golden_sytrf.py).
 *
 * Storage: column-major, lower triangle only (the strict upper triangle is
 * never read or written).  Output: L's multipliers below the diagonal, D's
 * 1x1 entries on the diagonal and each 2x2 block's off-diagonal at (k+1, k),
 * perm[pos] = original index at position pos, piv_size 1 / 2 (block start) /
 * 0 (second column of a 2x2 block, or delayed), info = start of the delayed
 * suffix, whose trailing block holds the Schur complement.  Each step follows
 * the reference line it cites; BLAS calls are plain loops. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

/* (1 + sqrt(17)) / 8 and 64 u, delayed_sytrf_blocked.cpp:21-25. */
static const double kAlpha = (1.0 + 4.1231056256176605498) / 8.0;
static const double kDetTol = 64.0 * 2.220446049250313080847e-16;

static double sym_lower(const double *a, int lda, int r, int c) { /* :29-32 */
  return r >= c ? a[IDX(r, c, lda)] : a[IDX(c, r, lda)];
}

static void dswap_strided(int n, double *x, int incx, double *y, int incy) {
  for (int i = 0; i < n; ++i) {
    double t = x[(size_t)i * incx];
    x[(size_t)i * incx] = y[(size_t)i * incy];
    y[(size_t)i * incy] = t;
  }
}

/* symmetric_swap_lower, delayed_sytrf_blocked.cpp:34-61: positions x and y
 * exchange places in the lower-stored matrix, perm follows. */
static void sym_swap(int n, double *a, int lda, int x, int y, int *perm) {
  if (x == y) return;
  if (x > y) { int t = x; x = y; y = t; }
  if (x > 0) dswap_strided(x, a + x, lda, a + y, lda);
  if (y - x - 1 > 0) dswap_strided(y - x - 1, a + IDX(x + 1, x, lda), 1, a + IDX(y, x + 1, lda), lda);
  double t = a[IDX(x, x, lda)];
  a[IDX(x, x, lda)] = a[IDX(y, y, lda)];
  a[IDX(y, y, lda)] = t;
  if (n - y - 1 > 0) dswap_strided(n - y - 1, a + IDX(y + 1, x, lda), 1, a + IDX(y + 1, y, lda), 1);
  int p = perm[x]; perm[x] = perm[y]; perm[y] = p;
}

/* swap_active_nodes, :63-73: the swap plus the rows of the W = L D panel. */
static void swap_nodes(int n, double *a, int lda, int x, int y, int *perm, double *w, int ldw,
                       int pw) {
  if (x == y) return;
  sym_swap(n, a, lda, x, y, perm);
  if (pw > 0) dswap_strided(pw, w + x, ldw, w + y, ldw);
}

/* materialize_current_column, :75-88: column `col` (rows col..n-1) of the
 * matrix with this panel's update applied, A(:,col) - L_panel W(col,:)^T.
 * `acc` (n doubles): each row's sum over the panel columns, accumulated in
 * column order j = 0, 1, ... with the rows contiguous in the inner loop. */
static void mat_column(int n, const double *a, int lda, int pb, int pw, const double *w, int ldw,
                       int col, double *out, double *acc) {
  for (int r = col; r < n; ++r) acc[r] = 0.0;
  for (int j = 0; j < pw; ++j) {
    const double wj = w[IDX(col, j, ldw)];
    const double *lj = a + IDX(0, pb + j, lda);
    for (int r = col; r < n; ++r) acc[r] += lj[r] * wj;
  }
  for (int r = col; r < n; ++r) out[r] = a[IDX(r, col, lda)] - acc[r];
}

/* materialize_active_row, :90-106: row `row` over the active columns
 * (sums accumulated as in mat_column). */
static void mat_row(const double *a, int lda, int pb, int pw, const double *w, int ldw, int b,
                    int e, int row, double *out, double *acc) {
  for (int c = b; c < e; ++c) acc[c] = 0.0;
  for (int j = 0; j < pw; ++j) {
    const double wj = w[IDX(row, j, ldw)];
    const double *lj = a + IDX(0, pb + j, lda);
    for (int c = b; c < e; ++c) acc[c] += lj[c] * wj;
  }
  for (int c = b; c < e; ++c) out[c] = sym_lower(a, lda, row, c) - acc[c];
}

/* stable_2x2, :108-124. */
static int stable_2x2(double a, double b, double c) {
  double s = fmax(fabs(a), fmax(fabs(b), fabs(c)));
  if (!(s > 0.0)) return 0;
  double as = a / s, bs = b / s, cs = c / s;
  double det = as * cs - bs * bs;
  double nrm = fmax(fabs(as) + fabs(bs), fabs(bs) + fabs(cs));
  return fabs(det) > kDetTol * nrm * nrm;
}

/* cblas_idamax: first index of the largest magnitude (a NaN never wins). */
static int first_absmax(int n, const double *x) {
  int best = 0;
  double bv = -1.0;
  for (int i = 0; i < n; ++i) {
    double v = fabs(x[i]);
    if (v > bv) { bv = v; best = i; }
  }
  return best;
}

/* finish_panel, :126-139: lower triangle of the trailing block minus
 * (L W^T + W L^T) / 2 over the panel's columns; per element the sum runs over
 * j = 0, 1, ... (rows contiguous in the inner loop, one sum array per
 * column). */
static void finish_panel(int n, double *a, int lda, int begin, int end, const double *w,
                         int ldw) {
  const int width = end - begin;
  if (width <= 0 || n - end <= 0) return;
#pragma omp parallel
  {
    double *acc = malloc(sizeof(double) * (size_t)n);
#pragma omp for schedule(dynamic, 16)
    for (int c = end; c < n; ++c) {
      if (!acc) continue;
      for (int r = c; r < n; ++r) acc[r] = 0.0;
      for (int j = 0; j < width; ++j) {
        const double wc = w[IDX(c, j, ldw)], ac = a[IDX(c, begin + j, lda)];
        const double *lj = a + IDX(0, begin + j, lda), *wj = w + IDX(0, j, ldw);
        for (int r = c; r < n; ++r) acc[r] += lj[r] * wc + wj[r] * ac;
      }
      for (int r = c; r < n; ++r) a[IDX(r, c, lda)] -= 0.5 * acc[r];
    }
    free(acc);
  }
}

/* delayed_sytrf_blocked, :141-358, with the panel width as a parameter
 * (the reference fixes kBlockSize = 64, :23).  Returns info. */
int oracle_sytrf(int n, double *a, int lda, int *perm, int *piv_size, int nb) {
  if (n < 0 || lda < (n > 1 ? n : 1) || nb < 2 || (n > 0 && (!a || !perm || !piv_size))) return -1;
  for (int i = 0; i < n; ++i) { perm[i] = i; piv_size[i] = 0; }
  if (n == 0) return 0;
  const int ldw = n;
  double *w = calloc((size_t)ldw * nb, sizeof(double));
  double *c0 = calloc((size_t)n, sizeof(double));
  double *c1 = calloc((size_t)n, sizeof(double));
  double *rv = calloc((size_t)n, sizeof(double));
  double *acc = calloc((size_t)n, sizeof(double));
  if (!w || !c0 || !c1 || !rv || !acc) {
    free(w); free(c0); free(c1); free(rv); free(acc);
    return -1;
  }

  int pb = 0, e = n;
  while (pb < e) {
    int k = pb, pw = 0;
    while (k < e && pw < nb) {
      mat_column(n, a, lda, pb, pw, w, ldw, k, c0, acc);
      const double akk = fabs(c0[k]);
      int p = k;
      double colmax = 0.0;
      if (e - k > 1) { /* :183-190 */
        p = k + 1 + first_absmax(e - k - 1, c0 + k + 1);
        colmax = fabs(c0[p]);
      }
      int one = 0, two = 0, piv = k;
      if (!(fmax(akk, colmax) > 0.0)) {
        /* both candidates zero: delay (:196-199) */
      } else if (akk >= kAlpha * colmax) {
        one = 1; /* criterion 1 (:200-202) */
      } else {
        mat_row(a, lda, pb, pw, w, ldw, k, e, p, rv, acc);
        double rowmax = 0.0;
        for (int c = k; c < e; ++c)
          if (c != p) rowmax = fmax(rowmax, fabs(rv[c]));
        const double app = fabs(rv[p]);
        if (akk >= kAlpha * colmax * (colmax / rowmax)) {
          one = 1; /* criterion 2 */
        } else if (app >= kAlpha * rowmax) {
          one = 1; piv = p; /* criterion 3 */
        } else if (stable_2x2(c0[k], c0[p], rv[p])) {
          two = 1; piv = p; /* 2x2 block (k, p) */
        }
      }
      if (!one && !two) { /* :237-243 — node k to the front of the delayed suffix */
        swap_nodes(n, a, lda, k, e - 1, perm, w, ldw, pw);
        --e;
        continue;
      }
      if (two && pw + 2 > nb) break; /* :245-248 — the block starts the next panel */
      if (one) { /* :250-272 */
        if (piv != k) {
          swap_nodes(n, a, lda, k, piv, perm, w, ldw, pw);
          mat_column(n, a, lda, pb, pw, w, ldw, k, c0, acc);
        }
        const double d = c0[k];
        a[IDX(k, k, lda)] = d;
        piv_size[k] = 1;
        w[IDX(k, pw, ldw)] = d;
        for (int r = k + 1; r < n; ++r) {
          a[IDX(r, k, lda)] = c0[r] / d;
          w[IDX(r, pw, ldw)] = c0[r];
        }
        ++k; ++pw;
        continue;
      }
      /* 2x2 block, :274-330 */
      swap_nodes(n, a, lda, k + 1, piv, perm, w, ldw, pw);
      mat_column(n, a, lda, pb, pw, w, ldw, k, c0, acc);
      mat_column(n, a, lda, pb, pw, w, ldw, k + 1, c1, acc);
      const double d00 = c0[k], d10 = c0[k + 1], d11 = c1[k + 1];
      a[IDX(k, k, lda)] = d00;
      a[IDX(k + 1, k, lda)] = d10;
      a[IDX(k + 1, k + 1, lda)] = d11;
      piv_size[k] = 2;
      piv_size[k + 1] = 0;
      const double s = fmax(fabs(d00), fmax(fabs(d10), fabs(d11)));
      const double s00 = d00 / s, s10 = d10 / s, s11 = d11 / s;
      const double inv = 1.0 / (s * (s00 * s11 - s10 * s10));
      w[IDX(k, pw, ldw)] = d00;
      w[IDX(k + 1, pw, ldw)] = d10;
      w[IDX(k, pw + 1, ldw)] = d10;
      w[IDX(k + 1, pw + 1, ldw)] = d11;
      for (int r = k + 2; r < n; ++r) {
        const double b0 = c0[r], b1 = c1[r];
        a[IDX(r, k, lda)] = (s11 * b0 - s10 * b1) * inv;
        a[IDX(r, k + 1, lda)] = (s00 * b1 - s10 * b0) * inv;
        w[IDX(r, pw, ldw)] = b0;
        w[IDX(r, pw + 1, ldw)] = b1;
      }
      k += 2;
      pw += 2;
    }
    finish_panel(n, a, lda, pb, k, w, ldw);
    pb = k;
  }
  free(w); free(c0); free(c1); free(rv); free(acc);
  return e;
}
