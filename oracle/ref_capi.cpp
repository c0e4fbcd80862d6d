// extern "C" shims over the reference's own CPU entry points, so that tests and
// the CPU arm of bench.py can call the compiled reference through ctypes.
//
// Test infrastructure only: built into oracle/_ref/ together with the
// reference's unmodified sources (delayed_lu/delayed_dgetrf.cpp,
// delayed_lu/delayed_dgetrf_column.cpp, delayed_lu/lapack_dgetrf.cpp) by
// oracle/Makefile.  Nothing in the product library links it.
#include "delayed_dgetrf.hpp"
#include "delayed_dgetrf_column.hpp"
#include "lapack_dgetrf.hpp"

extern "C" {
void scipy_openblas_set_num_threads(int);
int scipy_openblas_get_num_threads(void);

// delayed_lu/delayed_dgetrf.hpp:17 — full-pivot fallback.
void ref_delayed_getrf(int m, int n, double *a, int lda, int *ipiv, int *jpiv,
                       int *info) {
  int i = -1;
  delayed_getrf(m, n, a, lda, ipiv, jpiv, i);
  *info = i;
}

// delayed_lu/delayed_dgetrf_column.hpp — right-to-left nonzero-column fallback.
void ref_delayed_getrf_column(int m, int n, double *a, int lda, int *ipiv,
                              int *jpiv, int *info) {
  int i = -1;
  delayed_getrf_column(m, n, a, lda, ipiv, jpiv, i);
  *info = i;
}

// delayed_lu/lapack_dgetrf.hpp:6 — LAPACK dgetrf with 0-based ipiv.
void ref_lapack_getrf(int m, int n, double *a, int lda, int *ipiv, int *info) {
  int i = -1;
  lapack_getrf(m, n, a, lda, ipiv, i);
  *info = i;
}

void ref_set_threads(int t) { scipy_openblas_set_num_threads(t); }
int ref_get_threads(void) { return scipy_openblas_get_num_threads(); }
}
