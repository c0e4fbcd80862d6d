// Drop-in C++ interface of the B200 delayed-pivoting LU.
//
// Same declarations, argument meaning and error behaviour as the reference's
// delayed_lu_cuda/delayed_dgetrf_cuda.hpp:1-63, so callers written against it
// (delayed_lu_cuda/example.cu, delayed_lu_cuda/benchmark.cu) compile and link
// unchanged against libdelayed_lu_b200.so.
//
//  - A is column-major, 0-based, A(i,j) at a[i + j*lda], m x n, lda >= max(1,m);
//    it is overwritten in place with the compact L\U factors: strict lower part
//    of columns < info = L (unit diagonal implicit), rows < info from the
//    diagonal on = U, block [info:m, info:n] = the delayed Schur complement.
//  - ipiv / jpiv are HOST arrays of min(m,n) ints: the 0-based row / column
//    swapped with k at step k (a swap history; replay them in order to get P
//    and Q with P*A*Q = L*U).  Entries >= info stay identity.
//  - info = min(m,n) when no pivot was delayed, k when the active submatrix
//    from step k on holds no acceptable pivot, -1 when status != success.
//  - Every call is stream-ordered on `stream` and synchronises it before
//    returning.
#pragma once

#include <cuda_runtime_api.h>

enum class DelayedGetrfCudaStatus {
  success = 0,
  invalid_argument,
  allocation_failed,
  cuda_failure,
  cublas_failure,   // kept for ABI compatibility; this library never calls cuBLAS
  device_timeout,   // a bounded device-side wait gave up (no reference counterpart)
};

// delayed_dgetrf_cuda.hpp:24-26 — device-memory entry point.
DelayedGetrfCudaStatus delayed_getrf_cuda_device(int m, int n, double *d_a, int lda, int *ipiv,
                                                 int *jpiv, int &info,
                                                 cudaStream_t stream = nullptr);

// delayed_dgetrf_cuda.hpp:35-37 — host-memory convenience entry point: copies
// lda*n doubles to the GPU, factors them, copies the result back.
DelayedGetrfCudaStatus delayed_getrf_cuda_host(int m, int n, double *a, int lda, int *ipiv,
                                               int *jpiv, int &info,
                                               cudaStream_t stream = nullptr);

// delayed_dgetrf_cuda.hpp:40-46 — explicit "native" names.
DelayedGetrfCudaStatus delayed_getrf_cuda_native_device(int m, int n, double *d_a, int lda,
                                                        int *ipiv, int *jpiv, int &info,
                                                        cudaStream_t stream = nullptr);
DelayedGetrfCudaStatus delayed_getrf_cuda_native_host(int m, int n, double *a, int lda,
                                                      int *ipiv, int *jpiv, int &info,
                                                      cudaStream_t stream = nullptr);

// delayed_dgetrf_cuda.hpp:55-61 — the reference factors these panels on the
// CPU.  Here the panel never leaves the device: both names run the same
// device path as delayed_getrf_cuda_device / _host.
DelayedGetrfCudaStatus delayed_getrf_cuda_hybrid_device(int m, int n, double *d_a, int lda,
                                                        int *ipiv, int *jpiv, int &info,
                                                        cudaStream_t stream = nullptr);
DelayedGetrfCudaStatus delayed_getrf_cuda_hybrid_host(int m, int n, double *a, int lda,
                                                      int *ipiv, int *jpiv, int &info,
                                                      cudaStream_t stream = nullptr);

// delayed_dgetrf_cuda.hpp:63
const char *delayed_getrf_cuda_status_string(DelayedGetrfCudaStatus status);
