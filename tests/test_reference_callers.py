"""The reference's own callers of the drop-in header, unmodified
(delayed_lu_cuda/example.cu:113-162, delayed_lu_cuda/benchmark.cu:74-137),
compiled by oracle/Makefile against include/delayed_dgetrf_cuda.hpp and
libdelayed_lu_b200.so, and the reference's own cuBLAS build of the same
callers.  Exit code 77 is the callers' own "no GPU" skip."""
import re
import subprocess

import pytest

import oracle as orc


def _binary(name):
    p = orc.ref_binary(name)
    if p is None:
        pytest.skip(f"oracle/_ref/{name} not built (reference tree absent at build time)")
    return p


@pytest.mark.parametrize("name", ["example_on_b200", "benchmark_on_b200"])
def test_dropin_callers_link_this_library(name):
    """Without a GPU the callers load, resolve every symbol from
    libdelayed_lu_b200.so and take their own skip exit (77)."""
    p = _binary(name)
    ldd = subprocess.run(["ldd", str(p)], capture_output=True, text=True).stdout
    assert "libdelayed_lu_b200.so" in ldd and "not found" not in ldd
    assert "libcublas" not in ldd  # the drop-in needs no cuBLAS
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        r = subprocess.run([str(p)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 77, r.stdout + r.stderr


@pytest.mark.gpu
def test_reference_example_passes_on_this_library():
    """example.cu's four known-answer cases, through both the native and the
    hybrid entry points, pass on this library: info and the reconstruction
    tolerance 1e-11 max|A| max(m,n) (example.cu:105)."""
    r = subprocess.run([str(_binary("example_on_b200"))], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("PASS") == 8 and "FAIL" not in r.stdout, r.stdout


@pytest.mark.gpu
def test_reference_benchmark_runs_on_this_library():
    r = subprocess.run([str(_binary("benchmark_on_b200")), "1024", "2"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    rates = [float(x) for x in re.findall(r"([0-9.]+) GFLOP/s", r.stdout)]
    assert len(rates) == 2 and min(rates) > 0, r.stdout


@pytest.mark.gpu
def test_reference_own_cuda_example_on_b200():
    """The reference's own cuBLAS build runs its example on this GPU."""
    r = subprocess.run([str(_binary("ref_cuda_example"))], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout
