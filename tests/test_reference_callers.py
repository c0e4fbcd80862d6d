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


# ---- delayed Bunch-Kaufman: delayed-bunch-kaufman/example.cpp, unmodified ----

PASS_LINE = "总体比较结果：通过"  # the caller's own "overall comparison: pass" line


def test_bk_caller_links_this_library():
    """The reference's LDL^T caller, built against include/delayed_sytrf*.hpp,
    takes delayed_sytrf and delayed_sytrf_blocked from libdelayed_lu_b200.so
    (lapack_sytrf, the caller's comparison, from the reference's source)."""
    p = _binary("bk_example_on_b200")
    ldd = subprocess.run(["ldd", str(p)], capture_output=True, text=True).stdout
    assert "libdelayed_lu_b200.so" in ldd and "not found" not in ldd
    undef = subprocess.run(["nm", "-D", "--undefined-only", str(p)], capture_output=True,
                           text=True).stdout
    assert "_Z13delayed_sytrfiPdiPiS0_Ri" in undef
    assert "_Z21delayed_sytrf_blockediPdiPiS0_Ri" in undef


def test_bk_caller_passes_on_the_reference():
    """The same caller on the reference's CPU sources: its rank-8 known answer
    (info 8 for both delayed variants, reconstruction within 100 u rank)."""
    r = subprocess.run([str(_binary("bk_example_ref"))], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and PASS_LINE in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_bk_caller_passes_on_this_library():
    """The unmodified caller's known-answer check on the GPU path: info == 8
    from delayed_sytrf and delayed_sytrf_blocked, both reconstructions within
    100 u rank, LAPACK's as well."""
    r = subprocess.run([str(_binary("bk_example_on_b200"))], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and PASS_LINE in r.stdout, r.stdout + r.stderr
