"""ctypes bindings of the C ABI (include/delayed_pivoting_b200.h)."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent.parent
_LIB_DIR = _PKG / "lib"

SUCCESS, INVALID_ARGUMENT, ALLOCATION_FAILED, CUDA_FAILURE, LIBRARY_FAILURE, DEVICE_TIMEOUT = range(6)
POLICY_FULL_PIVOT, POLICY_NONZERO_COLUMN = 0, 1
PRECISION_FP64, PRECISION_MIXED_BF16X3 = 0, 1

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
        ("reserved", ctypes.c_int * 1),
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
                    precision=PRECISION_FP64):
    """dp_getrf_device_ex with explicit options.  Returns (status, info)."""
    opt = Options()
    lib().dp_options_init(ctypes.byref(opt))
    opt.nb, opt.threshold, opt.policy, opt.panel_rows = nb, threshold, policy, panel_rows
    opt.nb_outer = nb_outer
    opt.panel_kernel = panel_kernel
    opt.precision = precision
    info = ctypes.c_int(-1)
    st = lib().dp_getrf_device_ex(m, n, _dptr(d_a), lda, _iptr(ipiv), _iptr(jpiv),
                                  ctypes.byref(info), _stream(stream), ctypes.byref(opt))
    return st, info.value


def getrs_device(n, nrhs, d_lu, ldlu, ipiv, jpiv, d_b, ldb, stream=None):
    """dp_getrs_device: solve with the factors of getrf; d_b overwritten."""
    return lib().dp_getrs_device(n, nrhs, _dptr(d_lu), ldlu, _iptr(ipiv), _iptr(jpiv),
                                 _dptr(d_b), ldb, _stream(stream))


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
