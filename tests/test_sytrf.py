"""Delayed Bunch-Kaufman LDL^T (delayed-bunch-kaufman/): the restatement
(oracle/delayed_sytrf_oracle.c) pinned to the reference's own records, and
the GPU path (dp_sytrf_device) against both.

Records (perm, piv_size, info) are compared bit for bit; the factor values
through the reconstruction P A P^T = L D L^T of example.cpp:97-160 (the
delayed suffix's Schur complement as D's trailing block) and against the
restatement's factor."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

import oracle as orc

GOLDEN = Path(__file__).resolve().parent / "golden" / "sytrf"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load(name):
    g = np.load(GOLDEN / f"{name}.npz")
    n, lda = int(g["n"]), int(g["lda"])
    if bool(g["rank8"]):
        a = orc.rank8_example(n)
    else:
        a = orc.sym_matrix(n, int(g["seed"]), lda, tuple(int(z) for z in g["zero_nodes"]),
                           bool(g["zero_diag"]))
    return a, g


def test_package_generator_equals_oracle_generator():
    """bench.py builds its inputs with the package's generator, the fixtures
    with the oracle's: the two recipes must agree bit for bit."""
    import delayed_pivoting as dp

    for n, seed, lda, z, zd in ((7, 1, 7, (), False), (333, 7, 340, (40,), False),
                                (257, 6, 257, (0, 1, 2), True), (4096, 4096, 4096, (), False)):
        np.testing.assert_array_equal(dp.symmetric_matrix(n, seed, lda, z, zd),
                                      orc.sym_matrix(n, seed, lda, z, zd))


def test_fixtures_present():
    assert len(CASES) >= 15
    assert "rank8_4096" in CASES and "sym_4096" in CASES


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_records(name):
    a, g = load(name)
    f = a.copy(order="F")
    perm, piv, info = orc.oracle_sytrf(f)
    assert info == int(g["info"])
    np.testing.assert_array_equal(perm, g["perm"])
    np.testing.assert_array_equal(piv, g["piv_size"])
    err = orc.ldl_residual(a, f, perm, piv, info)
    assert err <= max(50 * float(g["max_error"]), 2e-13)


def test_rank8_known_answer():
    """example.cpp's check: info == rank == 8, one 2x2 block, exact factors."""
    a = orc.rank8_example(512)
    f = a.copy(order="F")
    perm, piv, info = orc.oracle_sytrf(f)
    assert info == 8
    assert int((piv == 2).sum()) == 1 and int((piv[:8] == 1).sum()) == 6
    assert orc.ldl_residual(a, f, perm, piv, info) <= 100 * np.finfo(float).eps * 8


@pytest.mark.parametrize("nb", [2, 3, 16, 64, 200])
def test_oracle_panel_width_keeps_records(nb):
    a, g = load("sym_300_zero2")
    perm, piv, info = orc.oracle_sytrf(a.copy(order="F"), nb=nb)
    assert info == int(g["info"])
    np.testing.assert_array_equal(perm, g["perm"])
    np.testing.assert_array_equal(piv, g["piv_size"])


def test_oracle_leaves_upper_triangle_and_padding():
    a, _ = load("sym_333_lda340")
    a[:, :] += np.triu(np.full(a.shape, 7.0), 1)  # junk above the diagonal
    a[333:, :] = -3.0                              # junk in the padding rows
    f = a.copy(order="F")
    orc.oracle_sytrf(f, n=333)
    np.testing.assert_array_equal(np.triu(f[:333], 1), np.triu(a[:333], 1))
    np.testing.assert_array_equal(f[333:], a[333:])


@pytest.mark.skipif(not orc.ref_bk_available(), reason="reference build absent")
@pytest.mark.parametrize("seed", [101, 102, 103])
def test_oracle_against_reference_on_fresh_inputs(seed):
    n = 97 + 31 * (seed - 100)
    a = orc.sym_matrix(n, seed, zero_nodes=(seed % n,), zero_diag=seed == 102)
    f, g = a.copy(order="F"), a.copy(order="F")
    r_or = orc.oracle_sytrf(f)
    r_ref = orc.ref_sytrf(g, "blocked")
    for x, y in zip(r_or[:2], r_ref[:2]):
        np.testing.assert_array_equal(x, y)
    assert r_or[2] == r_ref[2]
    assert np.abs(f - g).max() <= 1e-10 * max(1.0, np.abs(g).max())


@pytest.mark.skipif(not orc.ref_bk_available(), reason="reference build absent")
def test_oracle_against_reference_random_sweep():
    """60 seeded shapes (n 1..129, lda n..n+3, 0-3 zero nodes, 30 % with a
    cleared diagonal): the restatement's records equal the compiled
    reference's delayed_sytrf_blocked on every one."""
    rng = np.random.default_rng(5)
    for c in range(60):
        n = int(rng.integers(1, 130))
        lda = n + int(rng.integers(0, 4))
        z = tuple(sorted({int(x) for x in rng.integers(0, n, size=int(rng.integers(0, 4)))}))
        a = orc.sym_matrix(n, 1000 + c, lda, z, bool(rng.random() < 0.3))
        f, g = a.copy(order="F"), a.copy(order="F")
        r_or = orc.oracle_sytrf(f)
        r_ref = orc.ref_sytrf(g, "blocked")
        assert r_or[2] == r_ref[2], (c, n)
        np.testing.assert_array_equal(r_or[0], r_ref[0])
        np.testing.assert_array_equal(r_or[1], r_ref[1])


def test_c_abi_argument_checks_need_no_device():
    import delayed_pivoting as dp

    L = dp.lib()
    ip = ctypes.POINTER(ctypes.c_int)
    L.dp_sytrf_device.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ip, ip, ip,
                                  ctypes.c_void_p]
    perm = np.zeros(4, np.int32)
    piv = np.zeros(4, np.int32)
    info = ctypes.c_int(7)
    P = perm.ctypes.data_as(ip)
    Q = piv.ctypes.data_as(ip)
    assert L.dp_sytrf_device(-1, 0x1000, 1, P, Q, ctypes.byref(info), None) == dp.INVALID_ARGUMENT
    assert info.value == -1
    assert L.dp_sytrf_device(4, 0x1000, 3, P, Q, ctypes.byref(info), None) == dp.INVALID_ARGUMENT
    assert L.dp_sytrf_device(4, None, 4, P, Q, ctypes.byref(info), None) == dp.INVALID_ARGUMENT
    assert L.dp_sytrf_device(4, 0x1000, 4, None, Q, ctypes.byref(info), None) == dp.INVALID_ARGUMENT
    for nb in (1, 65, -5):
        st, *_ = dp.sytrf_device(4, 0x1000, 4, nb=nb)
        assert st == dp.INVALID_ARGUMENT
    assert dp.sytrf_device(4, 0x1000, 4, grid=-1)[0] == dp.INVALID_ARGUMENT
    st, _, _, info0 = dp.sytrf_device(0, None, 1)
    assert st == dp.SUCCESS and info0 == 0


def test_host_and_cxx_entry_points_reject_bad_arguments_without_a_device():
    """dp_sytrf_host and the C++ drop-in delayed_sytrf(_blocked) check their
    arguments before any device work; the drop-ins set info = -1 like the
    reference (delayed_sytrf.hpp:13)."""
    import delayed_pivoting as dp

    L = dp.lib()
    ip = ctypes.POINTER(ctypes.c_int)
    L.dp_sytrf_host.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ip, ip, ip]
    a = np.zeros((4, 4), order="F")
    perm = np.zeros(4, np.int32)
    piv = np.zeros(4, np.int32)
    info = ctypes.c_int(5)
    P, Q = perm.ctypes.data_as(ip), piv.ctypes.data_as(ip)
    assert L.dp_sytrf_host(-1, a.ctypes.data, 4, P, Q, ctypes.byref(info)) == dp.INVALID_ARGUMENT
    assert info.value == -1
    assert L.dp_sytrf_host(4, a.ctypes.data, 3, P, Q, ctypes.byref(info)) == dp.INVALID_ARGUMENT
    assert L.dp_sytrf_host(4, None, 4, P, Q, ctypes.byref(info)) == dp.INVALID_ARGUMENT
    for sym in ("_Z13delayed_sytrfiPdiPiS0_Ri", "_Z21delayed_sytrf_blockediPdiPiS0_Ri"):
        f = getattr(L, sym)
        f.restype = None
        f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ip, ip, ip]  # int& as pointer
        for n, lda in ((-1, 1), (4, 3)):
            info = ctypes.c_int(5)
            f(n, a.ctypes.data, lda, P, Q, ctypes.byref(info))
            assert info.value == -1, (sym, n, lda)


def test_cxx_drop_in_symbols_exported():
    import subprocess

    import delayed_pivoting as dp

    out = subprocess.run(["nm", "-D", str(dp.library_path())], capture_output=True, text=True).stdout
    assert "_Z13delayed_sytrfiPdiPiS0_Ri" in out          # delayed_sytrf(int, double*, int, int*, int*, int&)
    assert "_Z21delayed_sytrf_blockediPdiPiS0_Ri" in out  # delayed_sytrf_blocked(...)


# ---------------------------------------------------------------- GPU ----

def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _gpu_factor(a, **kw):
    import delayed_pivoting as dp

    torch = _torch()
    d = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()  # column-major storage of a
    st, perm, piv, info = dp.sytrf_device(a.shape[1], d, a.shape[0], **kw)
    rep = dp.sytrf_last_report()
    return st, perm, piv, info, np.asfortranarray(d.cpu().numpy().T), rep


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_records_match_reference(built, name):
    import delayed_pivoting as dp

    a, g = load(name)
    st, perm, piv, info, f, rep = _gpu_factor(a)
    assert st == dp.SUCCESS
    assert rep["near_ties"] == 0, rep
    assert info == int(g["info"])
    np.testing.assert_array_equal(perm, g["perm"])
    np.testing.assert_array_equal(piv, g["piv_size"])
    assert orc.ldl_residual(a, f, perm, piv, info) <= max(50 * float(g["max_error"]), 2e-13)
    # the same factor as the restatement, to rounding; the upper triangle untouched
    o = a.copy(order="F")
    orc.oracle_sytrf(o)
    n = a.shape[1]
    scale = max(1.0, float(np.abs(o[:n]).max()))
    assert np.abs(np.tril(f[:n] - o[:n])).max() <= 1e-10 * scale
    np.testing.assert_array_equal(np.triu(f[:n], 1), np.triu(a[:n], 1))
    np.testing.assert_array_equal(f[n:], a[n:])


@pytest.mark.gpu
def test_gpu_records_match_reference_n16384(built):
    """The seeded 16384 x 16384 symmetric matrix (2 GiB) against the
    reference's records (tests/golden/sytrf/large/sym_16384.npz, written by
    its delayed_sytrf_blocked; the restatement gives the same records), with
    no order-sensitive decision."""
    import delayed_pivoting as dp

    torch = _torch()
    g = np.load(GOLDEN / "large" / "sym_16384.npz")
    n = int(g["n"])
    a = dp.symmetric_matrix(n, int(g["seed"]))
    d = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    del a
    st, perm, piv, info = dp.sytrf_device(n, d, n)
    rep = dp.sytrf_last_report()
    del d
    torch.cuda.empty_cache()
    assert st == dp.SUCCESS and rep["near_ties"] == 0, rep
    assert info == int(g["info"])
    np.testing.assert_array_equal(perm, g["perm"])
    np.testing.assert_array_equal(piv, g["piv_size"])


@pytest.mark.gpu
@pytest.mark.parametrize("nb,grid", [(2, 0), (3, 4), (17, 8), (64, 5), (48, 0), (64, 148),
                                     (64, 16)])
def test_gpu_panel_width_and_grid_keep_records(built, nb, grid):
    """Panel widths 2..64 and CTA counts giving 1, 2 and 4 cached 128-row
    slots per CTA (grid 16, 8, 4 on n = 2048) keep the records."""
    a, g = load("sym_2048_zero8")
    st, perm, piv, info, f, rep = _gpu_factor(a, nb=nb, grid=grid)
    assert st == 0 and rep["near_ties"] == 0
    assert info == int(g["info"])
    np.testing.assert_array_equal(perm, g["perm"])
    np.testing.assert_array_equal(piv, g["piv_size"])


@pytest.mark.gpu
def test_gpu_rejects_grid_too_small_for_n(built):
    import delayed_pivoting as dp

    torch = _torch()
    d = torch.zeros(600, 600, dtype=torch.float64, device="cuda")
    assert dp.sytrf_device(600, d, 600, grid=1)[0] == dp.INVALID_ARGUMENT  # > 512 rows per CTA
    assert dp.sytrf_device(600, d, 600, grid=2)[0] == dp.SUCCESS


@pytest.mark.gpu
def test_gpu_host_entry_point_equals_device(built):
    import delayed_pivoting as dp

    a, g = load("zero_diag_257_zero3")
    h = a.copy(order="F")
    st, perm, piv, info = dp.sytrf_host(h)
    assert st == dp.SUCCESS and info == int(g["info"])
    np.testing.assert_array_equal(perm, g["perm"])
    np.testing.assert_array_equal(piv, g["piv_size"])
    _, _, _, _, f, _ = _gpu_factor(a)
    np.testing.assert_array_equal(h, f)


@pytest.mark.gpu
def test_gpu_large_reconstruction_and_report(built):
    """n = 6000 (panel kernel over 47 CTAs, 94 panels): reconstruction of a
    symmetric matrix with planted zero nodes, and a decision count equal to
    the factored columns plus the delays."""
    import delayed_pivoting as dp

    n = 6000
    zeros = (0, 17, 2999, 5998)
    a = orc.sym_matrix(n, 6000, zero_nodes=zeros)
    st, perm, piv, info, f, rep = _gpu_factor(a)
    assert st == dp.SUCCESS and info == n - len(zeros)
    assert sorted(perm[info:].tolist()) == sorted(zeros)
    steps = int((piv == 1).sum() + (piv == 2).sum()) + len(zeros)
    assert rep["decisions"] == steps and rep["info"] == info
    err = orc.ldl_residual(a, f, perm, piv, info)
    assert err <= 1e-11, err
