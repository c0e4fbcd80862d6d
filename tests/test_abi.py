"""CPU tests of the C ABI: the library loads, exports every symbol that
include/*.h declares (C and C++ drop-in names), and its argument checks
behave like the reference's (delayed_lu_cuda/delayed_dgetrf_cuda.cu:385-460)
without touching a GPU."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

# Itanium-mangled names of the reference header's C++ entry points
# (delayed_lu_cuda/delayed_dgetrf_cuda.hpp:24-63).
CXX_SYMBOLS = [
    "_Z25delayed_getrf_cuda_deviceiiPdiPiS0_RiP11CUstream_st",
    "_Z23delayed_getrf_cuda_hostiiPdiPiS0_RiP11CUstream_st",
    "_Z32delayed_getrf_cuda_native_deviceiiPdiPiS0_RiP11CUstream_st",
    "_Z30delayed_getrf_cuda_native_hostiiPdiPiS0_RiP11CUstream_st",
    "_Z32delayed_getrf_cuda_hybrid_deviceiiPdiPiS0_RiP11CUstream_st",
    "_Z30delayed_getrf_cuda_hybrid_hostiiPdiPiS0_RiP11CUstream_st",
    "_Z32delayed_getrf_cuda_status_string22DelayedGetrfCudaStatus",
]


def declared_c_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for mt in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(dp_\w+)\s*\(", text, flags=re.M):
            names.add(mt.group(1))
    return sorted(names)


def test_library_loads_and_exports_c_abi():
    import delayed_pivoting as dp

    L = dp.lib()
    names = declared_c_functions()
    assert "dp_getrf_device" in names and "dp_getrf_host" in names
    for name in names:
        assert hasattr(L, name), f"missing export {name}"


def test_library_exports_reference_cxx_symbols():
    import delayed_pivoting as dp

    out = subprocess.run(["nm", "-D", "--defined-only", str(dp.library_path())],
                         capture_output=True, text=True, check=True).stdout
    for sym in CXX_SYMBOLS:
        assert sym in out, sym


def test_header_declares_reference_entry_points():
    text = (ROOT / "include" / "delayed_dgetrf_cuda.hpp").read_text()
    for name in ("delayed_getrf_cuda_device", "delayed_getrf_cuda_host",
                 "delayed_getrf_cuda_native_device", "delayed_getrf_cuda_native_host",
                 "delayed_getrf_cuda_hybrid_device", "delayed_getrf_cuda_hybrid_host",
                 "delayed_getrf_cuda_status_string"):
        assert name in text


def test_status_strings():
    import delayed_pivoting as dp

    assert dp.delayed_getrf_cuda_status_string(0) == "success"
    assert dp.delayed_getrf_cuda_status_string(1) == "invalid argument"
    assert dp.delayed_getrf_cuda_status_string(2) == "CUDA allocation failed"
    assert dp.delayed_getrf_cuda_status_string(3) == "CUDA runtime failure"
    assert dp.delayed_getrf_cuda_status_string(4) == "cuBLAS failure"
    assert dp.delayed_getrf_cuda_status_string(5) == "device wait timed out"
    assert dp.delayed_getrf_cuda_status_string(99) == "unknown status"


@pytest.mark.parametrize("fn", ["delayed_getrf_cuda_device", "delayed_getrf_cuda_host"])
def test_invalid_arguments_rejected_before_any_device_work(fn):
    import delayed_pivoting as dp

    f = getattr(dp, fn)
    ipiv = np.zeros(4, dtype=np.int32)
    jpiv = np.zeros(4, dtype=np.int32)
    host = np.zeros((4, 4), order="F")
    a = host if fn.endswith("host") else 0x1000  # never dereferenced
    assert f(-1, 4, a, 4, ipiv, jpiv) == (dp.INVALID_ARGUMENT, -1)
    assert f(4, -1, a, 4, ipiv, jpiv) == (dp.INVALID_ARGUMENT, -1)
    assert f(4, 4, a, 3, ipiv, jpiv) == (dp.INVALID_ARGUMENT, -1)  # lda < m
    assert f(0, 0, a, 0, ipiv, jpiv) == (dp.INVALID_ARGUMENT, -1)  # lda < 1
    assert f(4, 4, None, 4, ipiv, jpiv) == (dp.INVALID_ARGUMENT, -1)
    assert f(4, 4, a, 4, None, jpiv) == (dp.INVALID_ARGUMENT, -1)
    assert f(4, 4, a, 4, ipiv, None) == (dp.INVALID_ARGUMENT, -1)


def test_empty_matrices_succeed_without_device_work():
    import delayed_pivoting as dp

    # pivots == 0: success, info = 0, no device access (delayed_dgetrf_cuda.cu:417-419, :456-460)
    assert dp.delayed_getrf_cuda_device(0, 5, None, 1, None, None) == (dp.SUCCESS, 0)
    assert dp.delayed_getrf_cuda_device(5, 0, None, 5, None, None) == (dp.SUCCESS, 0)
    assert dp.delayed_getrf_cuda_host(0, 0, None, 1, None, None) == (dp.SUCCESS, 0)


def test_options_rejected():
    import delayed_pivoting as dp

    ipiv = np.zeros(4, dtype=np.int32)
    jpiv = np.zeros(4, dtype=np.int32)
    assert dp.getrf_device_ex(4, 4, 0x1000, 4, ipiv, jpiv, threshold=-1.0) == (dp.INVALID_ARGUMENT, -1)
    assert dp.getrf_device_ex(4, 4, 0x1000, 4, ipiv, jpiv, threshold=float("nan")) == (dp.INVALID_ARGUMENT, -1)
    assert dp.getrf_device_ex(4, 4, 0x1000, 4, ipiv, jpiv, policy=7) == (dp.INVALID_ARGUMENT, -1)
    assert dp.getrf_device_ex(4, 4, 0x1000, 4, ipiv, jpiv, nb=-2) == (dp.INVALID_ARGUMENT, -1)


def test_package_exports_every_binding():
    """Every public function of delayed_pivoting.api is reachable from the
    package (the tests and bench.py call them as delayed_pivoting.<name>)."""
    import re
    from pathlib import Path

    import delayed_pivoting as dp

    src = (Path(dp.__file__).parent / "api.py").read_text()
    names = re.findall(r"^def ([a-z][a-z0-9_]*)\(", src, re.M)
    assert names
    assert [n for n in names if not hasattr(dp, n)] == []


def test_tuning_knobs_validate_and_restore():
    """The process-wide knobs reject values outside their range (returning the
    documented error value, leaving the setting unchanged) and return the
    previous setting; no device work is involved."""
    import delayed_pivoting as dp

    L = dp.lib()
    assert dp.block_solve(3) == -1 and dp.block_solve(-1) == -1
    prev = dp.block_solve(2)
    assert dp.block_solve(prev) == 2
    assert dp.mixed_gemm_grid(-2) == -2
    prev = dp.mixed_gemm_grid(-1)
    assert dp.mixed_gemm_grid(prev) == -1
    assert dp.gemm_tile(9) == -1
    prev = dp.gemm_tile(8)
    assert dp.gemm_tile(prev) == 8
    assert L.dp_tri_solve_grid(2000) == -2000
    prev = L.dp_tri_solve_grid(64)
    assert L.dp_tri_solve_grid(prev) == 64
