// Drop-in declaration of the reference's delayed_sytrf_blocked (delayed-bunch-kaufman/delayed_sytrf_blocked.hpp:15),
// implemented by libdelayed_lu_b200.so on the current GPU: the same
// signature and records (perm, piv_size, info), host memory in and out.
// Invalid arguments and device failures give info = -1.
#pragma once

void delayed_sytrf_blocked(int n, double *a, int lda, int *perm, int *piv_size, int &info);
