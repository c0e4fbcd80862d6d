// extern "C" shims over the reference's own CPU entry points of the delayed
// Bunch-Kaufman LDL^T, so that tests, the fixture generator and the CPU arm of
// bench.py can call the compiled reference through ctypes.
//
// Test infrastructure only: built into oracle/_ref/ together with the
// reference's unmodified sources (delayed-bunch-kaufman/delayed_sytrf.cpp,
// delayed_sytrf_blocked.cpp, lapack_dsytrf.cpp) by oracle/Makefile.  Nothing
// in the product library links it.
#include "delayed_sytrf.hpp"
#include "delayed_sytrf_blocked.hpp"
#include "lapack_dsytrf.hpp"

extern "C" {
void scipy_openblas_set_num_threads(int);

// delayed-bunch-kaufman/delayed_sytrf.hpp:15 — unblocked (dsyr / dsyr2 updates).
void ref_delayed_sytrf(int n, double *a, int lda, int *perm, int *piv_size, int *info) {
  int i = -1;
  delayed_sytrf(n, a, lda, perm, piv_size, i);
  *info = i;
}

// delayed-bunch-kaufman/delayed_sytrf_blocked.hpp:15 — W = L D panels of 64
// with a dsyr2k flush.
void ref_delayed_sytrf_blocked(int n, double *a, int lda, int *perm, int *piv_size,
                               int *info) {
  int i = -1;
  delayed_sytrf_blocked(n, a, lda, perm, piv_size, i);
  *info = i;
}

// delayed-bunch-kaufman/lapack_dsytrf.hpp — LAPACK dsytrf('L') + dsyconv,
// converted to the same perm / piv_size / explicit L, D layout.
void ref_lapack_sytrf(int n, double *a, int lda, int *perm, int *piv_size, int *info) {
  int i = -1;
  lapack_sytrf(n, a, lda, perm, piv_size, i);
  *info = i;
}

void ref_bk_set_threads(int t) { scipy_openblas_set_num_threads(t); }
}
