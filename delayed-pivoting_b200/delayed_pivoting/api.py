"""ctypes bindings of the C ABI (include/delayed_pivoting_b200.h)."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent.parent
_LIB_DIR = _PKG / "lib"

SUCCESS, INVALID_ARGUMENT, ALLOCATION_FAILED, CUDA_FAILURE, LIBRARY_FAILURE, DEVICE_TIMEOUT = range(6)
POLICY_FULL_PIVOT, POLICY_NONZERO_COLUMN = 0, 1
PRECISION_FP64, PRECISION_MIXED_BF16X3, PRECISION_MIXED_BF16X6 = 0, 1, 2
BATCH_MAX_N, BATCH_MAX_NB, BATCH_BUCKETS = 512, 32, 4

_lib = None
_gen = None


class Options(ctypes.Structure):
    """dp_options: panel width, acceptance threshold, fallback policy."""

    _fields_ = [
        ("nb", ctypes.c_int),
        ("threshold", ctypes.c_double),
        ("policy", ctypes.c_int),
        ("panel_rows", ctypes.c_int),
        ("nb_outer", ctypes.c_int),
        ("panel_kernel", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("lookahead", ctypes.c_int),
    ]


class IRResult(ctypes.Structure):
    """dp_ir_result of dp_gesv_ir_device."""

    _fields_ = [
        ("info", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("refactored", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("backward_error", ctypes.c_double),
        ("factor_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
    ]


class GetrfReport(ctypes.Structure):
    """dp_getrf_report: pivot decisions checked by the near-tie detector."""

    _fields_ = [
        ("decisions", ctypes.c_longlong),
        ("near_ties", ctypes.c_longlong),
        ("max_closeness", ctypes.c_double),
        ("info", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]

    def as_dict(self):
        return {"decisions": int(self.decisions), "near_ties": int(self.near_ties),
                "max_closeness": float(self.max_closeness), "info": int(self.info)}


class BatchOptions(ctypes.Structure):
    """dp_batch_options: threshold, precision, panel width per order bucket."""

    _fields_ = [
        ("threshold", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("nb_bucket", ctypes.c_int * BATCH_BUCKETS),
        ("reserved", ctypes.c_int * 2),
    ]


class ServerOptions(ctypes.Structure):
    """dp_server_options: HBM budget, precision, workers, batching, refinement."""

    _fields_ = [
        ("budget_bytes", ctypes.c_ulonglong),
        ("precision", ctypes.c_int),
        ("large_workers", ctypes.c_int),
        ("small_max_n", ctypes.c_int),
        ("small_max_batch", ctypes.c_int),
        ("max_iter", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("panel_rows", ctypes.c_int),
        ("mixed_min_n", ctypes.c_int),
        ("reserved", ctypes.c_int * 2),
    ]


class Request(ctypes.Structure):
    """dp_request: factor + solve (factor_id 0) or a follow-up solve."""

    _fields_ = [
        ("id", ctypes.c_ulonglong),
        ("factor_id", ctypes.c_ulonglong),
        ("n", ctypes.c_int),
        ("d_a", ctypes.c_void_p),
        ("lda", ctypes.c_int),
        ("d_b", ctypes.c_void_p),
        ("ldb", ctypes.c_int),
        ("nrhs", ctypes.c_int),
        ("followups", ctypes.c_int),
        ("reserved", ctypes.c_int),
    ]


class RequestResult(ctypes.Structure):
    """dp_request_result: status, info, precision, refinement, timestamps."""

    _fields_ = [
        ("id", ctypes.c_ulonglong),
        ("status", ctypes.c_int),
        ("info", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("refactored", ctypes.c_int),
        ("path", ctypes.c_int),
        ("backward_error", ctypes.c_double),
        ("t_submit", ctypes.c_double),
        ("t_admit", ctypes.c_double),
        ("t_start", ctypes.c_double),
        ("t_done", ctypes.c_double),
        ("factor_ms", ctypes.c_double),
        ("solve_ms", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("bytes_in_use", ctypes.c_ulonglong),
        ("bytes_peak", ctypes.c_ulonglong),
        ("submitted", ctypes.c_longlong),
        ("completed", ctypes.c_longlong),
        ("pending", ctypes.c_longlong),
        ("residents", ctypes.c_longlong),
        ("small_launches", ctypes.c_longlong),
        ("small_items", ctypes.c_longlong),
        ("large_items", ctypes.c_longlong),
    ]


def library_path() -> Path:
    return _LIB_DIR / "libdelayed_lu_b200.so"


def lib() -> ctypes.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        path = library_path()
        if not path.exists():
            raise RuntimeError(f"CUDA library not built: {path} (run __graft_entry__.build())")
        L = ctypes.CDLL(str(path))
        ip = ctypes.POINTER(ctypes.c_int)
        for name in ("dp_getrf_device", "dp_getrf_host", "dp_getrf_native_device",
                     "dp_getrf_native_host", "dp_getrf_hybrid_device", "dp_getrf_hybrid_host",
                     "dp_getrf_device_noalloc"):
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ip, ip, ip,
                          ctypes.c_void_p]
        L.dp_getrf_device_ex.restype = ctypes.c_int
        L.dp_getrf_device_ex.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                         ip, ip, ip, ctypes.c_void_p, ctypes.POINTER(Options)]
        L.dp_getrs_device.restype = ctypes.c_int
        L.dp_getrs_device.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                      ip, ip, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.dp_gesv_ir_device.restype = ctypes.c_int
        L.dp_gesv_ir_device.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.POINTER(IRResult), ctypes.c_void_p]
        L.dp_stats_enable.restype = None
        L.dp_stats_enable.argtypes = [ctypes.c_int]
        L.dp_stats_reset.restype = None
        L.dp_stats_reset.argtypes = []
        L.dp_status_string.restype = ctypes.c_char_p
        L.dp_status_string.argtypes = [ctypes.c_int]
        vp, ll = ctypes.c_void_p, ctypes.c_longlong
        bo = ctypes.POINTER(BatchOptions)
        L.dp_batch_options_init.restype = None
        L.dp_batch_options_init.argtypes = [bo]
        L.dp_batch_create.restype = ctypes.c_int
        L.dp_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp, vp, bo]
        L.dp_batch_layout.restype = ctypes.c_int
        L.dp_batch_layout.argtypes = [vp, vp, vp, ctypes.POINTER(ll), ctypes.POINTER(ll)]
        L.dp_batch_set_options.restype = ctypes.c_int
        L.dp_batch_set_options.argtypes = [vp, bo]
        for f in (L.dp_batch_getrf_async, L.dp_batch_getrf_graph):
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, vp, vp, vp, vp]
        L.dp_batch_destroy.restype = None
        L.dp_batch_destroy.argtypes = [vp]
        L.dp_batch_autotune.restype = ctypes.c_int
        L.dp_batch_autotune.argtypes = [bo, ctypes.c_int, ctypes.c_ulonglong, vp]
        L.dp_batch_tune_save.restype = ctypes.c_int
        L.dp_batch_tune_save.argtypes = [ctypes.c_char_p, bo]
        L.dp_batch_tune_load.restype = ctypes.c_int
        L.dp_batch_tune_load.argtypes = [ctypes.c_char_p, bo]
        L.dp_factor_create.restype = ctypes.c_int
        L.dp_factor_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp, ctypes.c_int,
                                       ctypes.c_int, vp]
        L.dp_factor_info.restype = ctypes.c_int
        L.dp_factor_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_double)]
        L.dp_factor_solve.restype = ctypes.c_int
        L.dp_factor_solve.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double, ctypes.POINTER(IRResult), vp]
        L.dp_factor_destroy.restype = None
        L.dp_factor_destroy.argtypes = [vp, vp]
        L.dp_server_options_init.restype = None
        L.dp_server_options_init.argtypes = [ctypes.POINTER(ServerOptions)]
        L.dp_server_create.restype = ctypes.c_int
        L.dp_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ServerOptions)]
        L.dp_server_submit.restype = ctypes.c_int
        L.dp_server_submit.argtypes = [vp, ctypes.POINTER(Request)]
        L.dp_server_poll.restype = ctypes.c_int
        L.dp_server_poll.argtypes = [vp, ctypes.POINTER(RequestResult), ctypes.c_int, ctypes.c_int]
        L.dp_server_stats_get.restype = ctypes.c_int
        L.dp_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.dp_server_clock.restype = ctypes.c_double
        L.dp_server_clock.argtypes = []
        L.dp_server_destroy.restype = None
        L.dp_server_destroy.argtypes = [vp]
        L.dp_options_init.restype = None
        L.dp_options_init.argtypes = [ctypes.POINTER(Options)]
        _lib = L
    return _lib


def matgen() -> ctypes.CDLL:
    global _gen
    if _gen is None:
        path = _LIB_DIR / "libdp_matgen.so"
        if not path.exists():
            raise RuntimeError(f"generator library not built: {path}")
        G = ctypes.CDLL(str(path))
        G.dpgen_mt64_nth.restype = ctypes.c_uint64
        G.dpgen_mt64_nth.argtypes = [ctypes.c_uint64, ctypes.c_int]
        G.dpgen_normal_matrix.restype = None
        G.dpgen_normal_matrix.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_longlong, ctypes.c_uint64]
        G.dpgen_normal_vector.restype = None
        G.dpgen_normal_vector.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_uint64]
        G.dpgen_plant_columns.restype = ctypes.c_int
        G.dpgen_plant_columns.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_longlong, ctypes.c_uint64, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p]
        G.dpgen_uniform.restype = None
        G.dpgen_uniform.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_uint64]
        _gen = G
    return _gen


def _iptr(arr):
    if arr is None:
        return None
    assert arr.dtype == np.int32 and arr.flags.c_contiguous
    return arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dptr(x):
    """Device pointer of a torch tensor, or an int address, or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _call(name, m, n, a_ptr, lda, ipiv, jpiv, stream):
    info = ctypes.c_int(-1)
    st = getattr(lib(), name)(m, n, a_ptr, lda, _iptr(ipiv), _iptr(jpiv), ctypes.byref(info),
                              _stream(stream))
    return st, info.value


def delayed_getrf_cuda_device(m, n, d_a, lda, ipiv, jpiv, stream=None):
    """delayed_dgetrf_cuda.hpp:24 — d_a device memory (torch tensor / address),
    ipiv/jpiv host int32 arrays of min(m,n).  Returns (status, info)."""
    return _call("dp_getrf_device", m, n, _dptr(d_a), lda, ipiv, jpiv, stream)


def delayed_getrf_cuda_host(m, n, a, lda, ipiv, jpiv, stream=None):
    """delayed_dgetrf_cuda.hpp:35 — a is a host float64 array (Fortran order,
    overwritten in place).  Returns (status, info)."""
    ptr = None if a is None else a.ctypes.data
    return _call("dp_getrf_host", m, n, ptr, lda, ipiv, jpiv, stream)


def delayed_getrf_cuda_native_device(m, n, d_a, lda, ipiv, jpiv, stream=None):
    return _call("dp_getrf_native_device", m, n, _dptr(d_a), lda, ipiv, jpiv, stream)


def delayed_getrf_cuda_native_host(m, n, a, lda, ipiv, jpiv, stream=None):
    return _call("dp_getrf_native_host", m, n, None if a is None else a.ctypes.data, lda, ipiv,
                 jpiv, stream)


def delayed_getrf_cuda_hybrid_device(m, n, d_a, lda, ipiv, jpiv, stream=None):
    return _call("dp_getrf_hybrid_device", m, n, _dptr(d_a), lda, ipiv, jpiv, stream)


def delayed_getrf_cuda_hybrid_host(m, n, a, lda, ipiv, jpiv, stream=None):
    return _call("dp_getrf_hybrid_host", m, n, None if a is None else a.ctypes.data, lda, ipiv,
                 jpiv, stream)


def delayed_getrf_cuda_status_string(status: int) -> str:
    return lib().dp_status_string(int(status)).decode()


def getrf_device_ex(m, n, d_a, lda, ipiv, jpiv, stream=None, nb=64, threshold=0.0,
                    policy=POLICY_FULL_PIVOT, panel_rows=0, nb_outer=0, panel_kernel=0,
                    precision=PRECISION_FP64, lookahead=0):
    """dp_getrf_device_ex with explicit options.  Returns (status, info).
    lookahead: 0 automatic, 1 on, 2 off (one stream, the unscheduled order)."""
    opt = Options()
    lib().dp_options_init(ctypes.byref(opt))
    opt.nb, opt.threshold, opt.policy, opt.panel_rows = nb, threshold, policy, panel_rows
    opt.nb_outer = nb_outer
    opt.panel_kernel = panel_kernel
    opt.precision = precision
    opt.lookahead = lookahead
    info = ctypes.c_int(-1)
    st = lib().dp_getrf_device_ex(m, n, _dptr(d_a), lda, _iptr(ipiv), _iptr(jpiv),
                                  ctypes.byref(info), _stream(stream), ctypes.byref(opt))
    return st, info.value


def getrf_autotune(n, stream=None):
    """dp_getrf_autotune: times the panel-width pairs for order n and records
    the fastest for n's order bucket; returns (status, nb, nb_outer)."""
    L = lib()
    L.dp_getrf_autotune.restype = ctypes.c_int
    L.dp_getrf_autotune.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    nb, nbo = ctypes.c_int(0), ctypes.c_int(0)
    st = L.dp_getrf_autotune(n, ctypes.byref(nb), ctypes.byref(nbo), _stream(stream))
    return st, nb.value, nbo.value


def getrf_tune_save(path) -> int:
    L = lib()
    L.dp_getrf_tune_save.restype = ctypes.c_int
    L.dp_getrf_tune_save.argtypes = [ctypes.c_char_p]
    return L.dp_getrf_tune_save(str(path).encode())


def getrf_tune_load(path) -> int:
    L = lib()
    L.dp_getrf_tune_load.restype = ctypes.c_int
    L.dp_getrf_tune_load.argtypes = [ctypes.c_char_p]
    return L.dp_getrf_tune_load(str(path).encode())


def getrf_last_report() -> dict:
    """dp_getrf_last_report: the near-tie report of this thread's last
    dp_getrf_* call (decisions, near_ties, max_closeness, info)."""
    L = lib()
    L.dp_getrf_last_report.restype = ctypes.c_int
    L.dp_getrf_last_report.argtypes = [ctypes.POINTER(GetrfReport)]
    r = GetrfReport()
    st = L.dp_getrf_last_report(ctypes.byref(r))
    if st != SUCCESS:
        raise RuntimeError(f"dp_getrf_last_report: status {st}")
    return r.as_dict()


def getrs_device(n, nrhs, d_lu, ldlu, ipiv, jpiv, d_b, ldb, stream=None):
    """dp_getrs_device: solve with the factors of getrf; d_b overwritten."""
    return lib().dp_getrs_device(n, nrhs, _dptr(d_lu), ldlu, _iptr(ipiv), _iptr(jpiv),
                                 _dptr(d_b), ldb, _stream(stream))


def schur_update_device(M, N, K, d_a, lda, d_b, ldb, d_c, ldc, stream=None):
    """dp_schur_update_device: C -= A * B in FP64 on the DMMA kernel
    (column-major operands; asynchronous on `stream`).  Returns the status."""
    L = lib()
    L.dp_schur_update_device.restype = ctypes.c_int
    L.dp_schur_update_device.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int] * 3 \
        + [ctypes.c_void_p]
    return L.dp_schur_update_device(M, N, K, _dptr(d_a), lda, _dptr(d_b), ldb, _dptr(d_c), ldc,
                                    _stream(stream))


def schur_update_mixed_device(M, N, K, d_a, lda, d_b, ldb, d_c, ldc,
                              precision=PRECISION_MIXED_BF16X6, stream=None):
    """dp_schur_update_mixed_device: C -= A * B on the tensor cores (BF16
    split, FP32 accumulation, C updated in FP64); synchronises.  Returns the
    status."""
    L = lib()
    L.dp_schur_update_mixed_device.restype = ctypes.c_int
    L.dp_schur_update_mixed_device.argtypes = [ctypes.c_int] * 3 + \
        [ctypes.c_void_p, ctypes.c_int] * 3 + [ctypes.c_int, ctypes.c_void_p]
    return L.dp_schur_update_mixed_device(M, N, K, _dptr(d_a), lda, _dptr(d_b), ldb, _dptr(d_c),
                                          ldc, precision, _stream(stream))


def gemm_tile(tile: int) -> int:
    """dp_gemm_tile: 0 automatic (= 5), 1 128 x 128, 2 128 x 64, 3 64 x 64, 4 128 x 64
    (8 warps), 5 64 x 64 (two stages), 6 64 x 128 (4 warps), 7 64 x 128 (8 warps),
    8 64 x 64 (32-deep k chunks).

    Returns the previous setting."""
    return lib().dp_gemm_tile(int(tile))


def front_factor(m, n, p, d_f, ldf, row_index=None, col_index=None, stream=None):
    """dp_front_factor: partial delayed LU of a frontal matrix whose leading p
    rows and columns are fully summed (multifrontal hand-off).  row_index /
    col_index: int32 arrays of the front's global indices (permuted in place).
    Returns (status, npiv, ipiv, jpiv); F(npiv:m, npiv:n) is then the
    contribution block, indexed by row_index[npiv:] and col_index[npiv:]."""
    L = lib()
    ip = ctypes.POINTER(ctypes.c_int)
    L.dp_front_factor.restype = ctypes.c_int
    L.dp_front_factor.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_int, ip, ip, ip, ip, ip, ctypes.c_void_p]
    ipiv = np.zeros(max(p, 1), dtype=np.int32)
    jpiv = np.zeros(max(p, 1), dtype=np.int32)
    k = ctypes.c_int(-1)
    st = L.dp_front_factor(m, n, p, _dptr(d_f), ldf, _iptr(row_index), _iptr(col_index),
                           _iptr(ipiv), _iptr(jpiv), ctypes.byref(k), _stream(stream))
    return st, k.value, ipiv[:p], jpiv[:p]


def extend_add(mc, nc, d_c, ldc, d_prow, d_pcol, d_p, ldp, stream=None) -> int:
    """dp_extend_add: P(prow[i], pcol[j]) += C(i, j) (device arrays; prow /
    pcol int32 positions in the parent)."""
    L = lib()
    vp = ctypes.c_void_p
    L.dp_extend_add.restype = ctypes.c_int
    L.dp_extend_add.argtypes = [ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp, vp, vp,
                                ctypes.c_int, vp]
    return L.dp_extend_add(mc, nc, _dptr(d_c), ldc, _dptr(d_prow), _dptr(d_pcol), _dptr(d_p),
                           ldp, _stream(stream))


class SytrfOptions(ctypes.Structure):
    """dp_sytrf_options: panel width (0 = 64) and panel-kernel CTAs (0 = automatic)."""

    _fields_ = [("nb", ctypes.c_int), ("grid", ctypes.c_int), ("reserved", ctypes.c_int * 6)]


def sytrf_device(n, d_a, lda, nb=0, grid=0, stream=None):
    """dp_sytrf_device_ex: delayed Bunch-Kaufman LDL^T of the symmetric matrix
    at d_a (device, column-major, lower triangle) in place - the GPU form of
    the reference's delayed_sytrf_blocked.  Returns (status, perm, piv_size,
    info)."""
    L = lib()
    ip = ctypes.POINTER(ctypes.c_int)
    L.dp_sytrf_device_ex.restype = ctypes.c_int
    L.dp_sytrf_device_ex.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ip, ip, ip,
                                     ctypes.POINTER(SytrfOptions), ctypes.c_void_p]
    perm = np.zeros(max(n, 1), dtype=np.int32)
    piv = np.zeros(max(n, 1), dtype=np.int32)
    info = ctypes.c_int(-1)
    opt = SytrfOptions(int(nb), int(grid))
    st = L.dp_sytrf_device_ex(n, _dptr(d_a), lda, _iptr(perm), _iptr(piv), ctypes.byref(info),
                              ctypes.byref(opt), _stream(stream))
    return st, perm[:max(n, 0)], piv[:max(n, 0)], info.value


def sytrf_host(a):
    """dp_sytrf_host on a Fortran-ordered float64 array (lda = a.shape[0]),
    factored in place through the GPU.  Returns (status, perm, piv_size, info)."""
    assert a.dtype == np.float64 and a.flags.f_contiguous
    L = lib()
    ip = ctypes.POINTER(ctypes.c_int)
    L.dp_sytrf_host.restype = ctypes.c_int
    L.dp_sytrf_host.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ip, ip, ip]
    n = a.shape[1]
    perm = np.zeros(max(n, 1), dtype=np.int32)
    piv = np.zeros(max(n, 1), dtype=np.int32)
    info = ctypes.c_int(-1)
    st = L.dp_sytrf_host(n, a.ctypes.data, a.shape[0], _iptr(perm), _iptr(piv),
                         ctypes.byref(info))
    return st, perm[:n], piv[:n], info.value


def sytrf_last_report() -> dict:
    """dp_sytrf_last_report: near-tie report of this thread's last dp_sytrf_* call."""
    L = lib()
    L.dp_sytrf_last_report.restype = ctypes.c_int
    L.dp_sytrf_last_report.argtypes = [ctypes.POINTER(GetrfReport)]
    r = GetrfReport()
    if L.dp_sytrf_last_report(ctypes.byref(r)) != SUCCESS:
        raise RuntimeError("dp_sytrf_last_report failed")
    return r.as_dict()


def mixed_gemm_grid(policy: int) -> int:
    """dp_mixed_gemm_grid: CTAs of the tensor-core update, 0 automatic (one per
    tile), g > 0 at most g, -1 one per SM (persistent).  Returns the previous setting."""
    return lib().dp_mixed_gemm_grid(int(policy))


def block_solve(mode: int) -> int:
    """dp_block_solve: triangular solves of the outer blocks, 0 automatic (= 1),
    1 by inverse (one FP64 tensor-core GEMM per block), 2 by substitution.

    Returns the previous setting."""
    return lib().dp_block_solve(int(mode))


def gesv_ir_device(n, nrhs, d_a, lda, d_b, ldb, precision=PRECISION_MIXED_BF16X3, max_iter=10,
                   tol=1e-14, stream=None):
    """dp_gesv_ir_device: mixed-precision LU + FP64 iterative refinement.
    Returns (status, IRResult)."""
    res = IRResult()
    st = lib().dp_gesv_ir_device(n, nrhs, _dptr(d_a), lda, _dptr(d_b), ldb, precision, max_iter,
                                 tol, ctypes.byref(res), _stream(stream))
    return st, res


def getrf_device_noalloc(m, n, d_a, lda, ipiv, jpiv, stream=None):
    """dp_getrf_device_noalloc: dp_getrf_device without any device allocation
    (scratch in a fixed array inside the library).  Returns (status, info)."""
    return _call("dp_getrf_device_noalloc", m, n, _dptr(d_a), lda, ipiv, jpiv, stream)


# ---- batched factorisation (dp_batch_*) -------------------------------------

def batch_options(threshold=0.0, nb_bucket=None, precision=PRECISION_FP64) -> BatchOptions:
    opt = BatchOptions()
    lib().dp_batch_options_init(ctypes.byref(opt))
    opt.threshold = threshold
    opt.precision = precision
    if nb_bucket is not None:
        if isinstance(nb_bucket, int):
            nb_bucket = [nb_bucket] * BATCH_BUCKETS
        for i, v in enumerate(nb_bucket):
            opt.nb_bucket[i] = int(v)
    return opt


class BatchError(RuntimeError):
    def __init__(self, status, what):
        super().__init__(f"{what}: status {status}")
        self.status = status


class Batch:
    """A dp_batch plan: the orders of a batch of square matrices, their
    layout in one device buffer, and the device work queue of the persistent
    kernel.  Matrix i is column-major with lda = n[i] at element offset
    ``offsets[i]``; its records are the n[i] entries at ``record_offsets[i]``
    of the device ipiv / jpiv arrays, its info ``info[i]``."""

    def __init__(self, ns, offsets=None, options: BatchOptions | None = None):
        self._h = None
        self.ns = np.ascontiguousarray(ns, dtype=np.int32)
        off = None if offsets is None else np.ascontiguousarray(offsets, dtype=np.int64)
        h = ctypes.c_void_p()
        st = lib().dp_batch_create(ctypes.byref(h), len(self.ns), self.ns.ctypes.data,
                                   None if off is None else off.ctypes.data,
                                   None if options is None else ctypes.byref(options))
        if st != SUCCESS:
            raise BatchError(st, "dp_batch_create")
        self._h = h
        n = len(self.ns)
        self.offsets = np.zeros(n, dtype=np.int64)
        self.record_offsets = np.zeros(n, dtype=np.int64)
        te, tr = ctypes.c_longlong(), ctypes.c_longlong()
        lib().dp_batch_layout(h, self.offsets.ctypes.data, self.record_offsets.ctypes.data,
                              ctypes.byref(te), ctypes.byref(tr))
        self.total_elements, self.total_records = te.value, tr.value

    def set_options(self, options: BatchOptions) -> int:
        return lib().dp_batch_set_options(self._h, ctypes.byref(options))

    def getrf_async(self, d_base, d_ipiv, d_jpiv, d_info, stream=None) -> int:
        return lib().dp_batch_getrf_async(self._h, _dptr(d_base), _dptr(d_ipiv), _dptr(d_jpiv),
                                          _dptr(d_info), _stream(stream))

    def getrf_graph(self, d_base, d_ipiv, d_jpiv, d_info, stream=None) -> int:
        return lib().dp_batch_getrf_graph(self._h, _dptr(d_base), _dptr(d_ipiv), _dptr(d_jpiv),
                                          _dptr(d_info), _stream(stream))

    def last_report(self) -> dict:
        """dp_batch_last_report: near-tie counts summed over the last launch
        (synchronises the device)."""
        L = lib()
        L.dp_batch_last_report.restype = ctypes.c_int
        L.dp_batch_last_report.argtypes = [ctypes.c_void_p, ctypes.POINTER(GetrfReport)]
        r = GetrfReport()
        st = L.dp_batch_last_report(self._h, ctypes.byref(r))
        if st != SUCCESS:
            raise BatchError(st, "dp_batch_last_report")
        return r.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            lib().dp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_autotune(options: BatchOptions | None = None, samples=12, seed=2024, stream=None):
    """dp_batch_autotune: returns (status, options with the tuned widths)."""
    opt = options if options is not None else batch_options()
    st = lib().dp_batch_autotune(ctypes.byref(opt), samples, seed, _stream(stream))
    return st, opt


def batch_tune_save(path, options: BatchOptions) -> int:
    return lib().dp_batch_tune_save(str(path).encode(), ctypes.byref(options))


def batch_tune_load(path, options: BatchOptions | None = None):
    opt = options if options is not None else batch_options()
    st = lib().dp_batch_tune_load(str(path).encode(), ctypes.byref(opt))
    return st, opt


# ---- resident factors (dp_factor_*) ----------------------------------------

class Factor:
    """dp_factor: a factorisation kept on the device for repeated refined solves."""

    def __init__(self, n, d_a, lda, precision=PRECISION_MIXED_BF16X3, stream=None):
        self._h = None
        h = ctypes.c_void_p()
        st = lib().dp_factor_create(ctypes.byref(h), n, _dptr(d_a), lda, precision,
                                    _stream(stream))
        if st != SUCCESS:
            raise BatchError(st, "dp_factor_create")
        self._h, self.n, self.d_a, self.lda = h, n, d_a, lda

    def info(self):
        """(info, precision of the factors held now, factorisation ms so far)."""
        i, p, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        lib().dp_factor_info(self._h, ctypes.byref(i), ctypes.byref(p), ctypes.byref(ms))
        return i.value, p.value, ms.value

    def solve(self, d_b, ldb, nrhs, max_iter=10, tol=1e-14, stream=None):
        """Overwrites d_b with X; returns (status, IRResult)."""
        res = IRResult()
        st = lib().dp_factor_solve(self._h, _dptr(self.d_a), self.lda, _dptr(d_b), ldb, nrhs,
                                   max_iter, tol, ctypes.byref(res), _stream(stream))
        return st, res

    def condest(self, stream=None):
        """dp_factor_condest: Hager-Higham estimate of kappa_1(A); returns
        (status, kappa1)."""
        L = lib()
        L.dp_factor_condest.restype = ctypes.c_int
        L.dp_factor_condest.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
        k = ctypes.c_double()
        st = L.dp_factor_condest(self._h, _dptr(self.d_a), self.lda, ctypes.byref(k),
                                 _stream(stream))
        return st, k.value

    def close(self, stream=None):
        if getattr(self, "_h", None):
            lib().dp_factor_destroy(self._h, _stream(stream))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- serving (dp_server_*) ---------------------------------------------------

def server_options(**kw) -> ServerOptions:
    opt = ServerOptions()
    lib().dp_server_options_init(ctypes.byref(opt))
    for k, v in kw.items():
        setattr(opt, k, v)
    return opt


def server_clock() -> float:
    return lib().dp_server_clock()


class Server:
    """dp_server: admits factor+solve requests and follow-up solves against an
    HBM budget and runs them overlapped on the current GPU."""

    def __init__(self, options: ServerOptions | None = None, **kw):
        self._h = None
        opt = options if options is not None else server_options(**kw)
        h = ctypes.c_void_p()
        st = lib().dp_server_create(ctypes.byref(h), ctypes.byref(opt))
        if st != SUCCESS:
            raise BatchError(st, "dp_server_create")
        self._h, self.options = h, opt

    def submit(self, rid, n, d_a, lda, d_b, ldb, nrhs, followups=0, factor_id=0) -> int:
        r = Request(id=rid, factor_id=factor_id, n=n, d_a=_dptr(d_a), lda=lda, d_b=_dptr(d_b),
                    ldb=ldb, nrhs=nrhs, followups=followups)
        return lib().dp_server_submit(self._h, ctypes.byref(r))

    def poll(self, max_results=256, wait_ms=0):
        buf = (RequestResult * max_results)()
        k = lib().dp_server_poll(self._h, buf, max_results, wait_ms)
        return [buf[i] for i in range(k)]

    def stats(self) -> ServerStats:
        s = ServerStats()
        lib().dp_server_stats_get(self._h, ctypes.byref(s))
        return s

    def close(self):
        if getattr(self, "_h", None):
            lib().dp_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
