"""GPU parity tests of the delayed-pivoting LU through the C ABI.

Records (ipiv, jpiv, info) must equal the reference's bit for bit (golden
fixtures from its own CPU code, tests/golden/); the factor must satisfy
||PAQ - LU||_F / (||A||_F * max(m,n) * u) <= 10.  Inputs that differ from the
fixtures (threshold > 0, other panel widths) are checked against the oracle
(oracle/delayed_getrf_oracle.c) on the same seeded input."""
import numpy as np
import pytest

import golden_cases as gc

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def assert_no_near_ties(info):
    """The near-tie detector saw every pivot decision of the last call and
    none of them was order-sensitive, so a records match is not luck."""
    import delayed_pivoting as dp

    rep = dp.getrf_last_report()
    assert rep["info"] == info
    assert rep["near_ties"] == 0, rep
    assert rep["decisions"] >= info, rep
    assert 0.0 <= rep["max_closeness"] < 1.0 or info == 0, rep
    return rep


def run_device(a, m, n, **opts):
    """Factors a (host Fortran array) on the GPU through dp_getrf_device[_ex];
    returns (factor (host), ipiv, jpiv, info, status)."""
    import delayed_pivoting as dp

    torch = _torch()
    lda = a.shape[0]
    d = torch.from_numpy(a.T.copy()).cuda()  # (n, lda) row-major == column-major lda x n
    k = max(min(m, n), 1)
    ipiv = np.full(k, -7, dtype=np.int32)
    jpiv = np.full(k, -7, dtype=np.int32)
    if opts:
        st, info = dp.getrf_device_ex(m, n, d, lda, ipiv, jpiv, **opts)
    else:
        st, info = dp.delayed_getrf_cuda_device(m, n, d, lda, ipiv, jpiv)
    torch.cuda.synchronize()
    fac = np.asfortranarray(d.cpu().numpy().T)
    kk = min(m, n)
    return fac, ipiv[:kk], jpiv[:kk], info, st


@pytest.mark.parametrize("name", gc.names(max_elems=4096 * 4096))
def test_records_match_reference(built, name):
    import oracle as orc

    a, case = gc.load(name)
    m, n = case["m"], case["n"]
    opts = {"policy": case["policy"]} if case["policy"] else {}
    fac, ipiv, jpiv, info, st = run_device(a, m, n, **opts)
    assert st == 0
    assert info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])
    assert_no_near_ties(info)
    assert orc.scaled_residual(a, fac, m, n, info, ipiv, jpiv) <= 10.0
    if case["lda"] > m:  # padding rows below m are never touched
        np.testing.assert_array_equal(fac[m:, :], a[m:, :])


def test_delayed_block_is_exactly_zero(built):
    a, case = gc.load("config1_n1024")
    fac, ipiv, jpiv, info, st = run_device(a, 1024, 1024)
    assert st == 0 and info == 1020
    assert np.all(fac[info:, info:] == 0.0)


@pytest.mark.parametrize("nb", [1, 8, 32, 100, 128])
def test_panel_width_does_not_change_records(built, nb):
    import oracle as orc

    a, case = gc.load("square_2000_zero20")
    fac, ipiv, jpiv, info, st = run_device(a, 2000, 2000, nb=nb)
    assert st == 0 and info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])
    assert_no_near_ties(info)
    assert orc.scaled_residual(a, fac, 2000, 2000, info, ipiv, jpiv) <= 10.0


@pytest.mark.parametrize("rows", [1, 7, 64, 1000])
def test_panel_cta_split_does_not_change_records(built, rows):
    a, case = gc.load("square_517_lda520")
    _, ipiv, jpiv, info, st = run_device(a, 517, 517, panel_rows=rows)
    assert st == 0 and info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])


@pytest.mark.parametrize("thr", [1e-14, 1e-9])
def test_threshold_matches_oracle(built, thr):
    import oracle as orc

    a, _ = gc.load("config1_n1024")
    o = a.copy(order="F")
    oi, oj, oinfo = orc.oracle_getrf(o, threshold=thr)
    fac, ipiv, jpiv, info, st = run_device(a, 1024, 1024, threshold=thr)
    assert st == 0 and info == oinfo == 1004
    np.testing.assert_array_equal(ipiv, oi)
    np.testing.assert_array_equal(jpiv, oj)
    assert np.abs(fac[info:, info:]).max() <= thr


@pytest.mark.parametrize("name", ["ref_dense_4x4", "ref_far_pivot_70", "tall_300x200",
                                  "wide_150x260"])
@pytest.mark.parametrize("entry", ["delayed_getrf_cuda_host", "delayed_getrf_cuda_native_host",
                                   "delayed_getrf_cuda_hybrid_host"])
def test_host_entry_points(built, name, entry):
    import delayed_pivoting as dp
    import oracle as orc

    _torch()
    a, case = gc.load(name)
    m, n = case["m"], case["n"]
    f = a.copy(order="F")
    k = min(m, n)
    ipiv = np.zeros(k, dtype=np.int32)
    jpiv = np.zeros(k, dtype=np.int32)
    st, info = getattr(dp, entry)(m, n, f, case["lda"], ipiv, jpiv)
    assert st == 0 and info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])
    assert orc.scaled_residual(a, f, m, n, info, ipiv, jpiv) <= 10.0


def test_device_aliases_and_user_stream(built):
    import delayed_pivoting as dp

    torch = _torch()
    a, case = gc.load("square_517_lda520")
    s = torch.cuda.Stream()
    for entry in ("delayed_getrf_cuda_native_device", "delayed_getrf_cuda_hybrid_device"):
        d = torch.from_numpy(a.T.copy()).cuda()
        ipiv = np.zeros(517, dtype=np.int32)
        jpiv = np.zeros(517, dtype=np.int32)
        torch.cuda.synchronize()
        st, info = getattr(dp, entry)(517, 517, d, 520, ipiv, jpiv, stream=s)
        assert st == 0 and info == case["info"]
        np.testing.assert_array_equal(ipiv, case["ipiv"])
        np.testing.assert_array_equal(jpiv, case["jpiv"])


def test_repeat_calls_are_deterministic(built):
    a, _ = gc.load("square_2000_zero20")
    f1 = run_device(a, 2000, 2000)[0]
    f2 = run_device(a, 2000, 2000)[0]
    np.testing.assert_array_equal(f1, f2)


@pytest.mark.parametrize("name,nb,nb_outer,panel", [
    ("square_2000_zero20", 64, 256, 0),   # fallback stops and restarts
    ("square_2000_zero20", 16, 48, 0),    # many blocks, restarts inside them
    ("square_2000_zero20", 16, 48, 2),    # grid-wide panel: one round trip per panel
    ("config1_n1024", 32, 96, 0),         # delays at the end
    ("tall_300x200", 8, 24, 0),
    ("wide_150x260", 8, 40, 0),           # columns right of the pivots
    ("square_517_lda520", 24, 64, 0),
])
def test_lookahead_changes_no_bit(built, name, nb, nb_outer, panel):
    """The look-ahead schedule (two streams, deferred row swaps, panels
    enqueued without a round trip and skipped on the device after a stop)
    gives every element the same operations in the same order as the
    one-stream order."""
    a, case = gc.load(name)
    m, n = case["m"], case["n"]
    kw = dict(nb=nb, nb_outer=nb_outer, policy=case["policy"], panel_kernel=panel)
    f1, i1, j1, info1, st1 = run_device(a, m, n, lookahead=1, **kw)
    f2, i2, j2, info2, st2 = run_device(a, m, n, lookahead=2, **kw)
    assert st1 == 0 and st2 == 0 and info1 == info2 == case["info"]
    np.testing.assert_array_equal(i1, case["ipiv"])
    np.testing.assert_array_equal(j1, case["jpiv"])
    np.testing.assert_array_equal(i1, i2)
    np.testing.assert_array_equal(j1, j2)
    np.testing.assert_array_equal(f1, f2)


def test_lookahead_mixed_precision_records(built):
    """Mixed precision: the next block's columns take their update in FP64
    under look-ahead, so factors differ in rounding only; records do not."""
    import oracle as orc

    a, case = gc.load("square_2000_zero20")
    kw = dict(nb=32, nb_outer=128, precision=2)
    f1, i1, j1, info1, st1 = run_device(a, 2000, 2000, lookahead=1, **kw)
    f2, i2, j2, info2, st2 = run_device(a, 2000, 2000, lookahead=2, **kw)
    assert st1 == 0 and st2 == 0 and info1 == info2 == case["info"]
    np.testing.assert_array_equal(i1, i2)
    np.testing.assert_array_equal(j1, j2)
    np.testing.assert_array_equal(i1, case["ipiv"])
    r1, an = orc.residual(a, f1, 2000, 2000, info1, i1, j1)
    r2, _ = orc.residual(a, f2, 2000, 2000, info2, i2, j2)
    assert r1 / an <= 1e-4  # FP32-level products with FP32 accumulation
    assert r1 <= 2.0 * r2  # FP64 on the next block's columns loses nothing


@pytest.mark.parametrize("M,N,K", [(1000, 300, 256), (517, 33, 24), (129, 70, 5), (64, 20, 64)])
def test_schur_update_against_torch(built, M, N, K):
    """C -= A B on the DMMA kernel: within FP64 rounding of torch's product,
    and bit-identical across tiles (each element accumulated in k order)."""
    import delayed_pivoting as dp

    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    lda, ldb, ldc = M + 3, K + 1, M + 5
    A = torch.randn(K, lda, dtype=torch.float64, device="cuda", generator=g)  # column-major
    B = torch.randn(N, ldb, dtype=torch.float64, device="cuda", generator=g)
    C0 = torch.randn(N, ldc, dtype=torch.float64, device="cuda", generator=g)
    ref = C0[:, :M].T - A[:, :M].T @ B[:, :K].T
    outs = []
    prev = dp.gemm_tile(0)
    try:
        for tile in (1, 2, 3, 4, 5):
            dp.gemm_tile(tile)
            C = C0.clone()
            torch.cuda.synchronize()
            assert dp.schur_update_device(M, N, K, A, lda, B, ldb, C, ldc) == 0
            torch.cuda.synchronize()
            assert torch.equal(C[:, M:], C0[:, M:])  # rows beyond M untouched
            outs.append(C[:, :M].T.clone())
    finally:
        dp.gemm_tile(prev)
    err = (outs[0] - ref).abs().max().item()
    assert err <= 1e-13 * K * max(1.0, ref.abs().max().item())
    for o in outs[1:]:
        assert torch.equal(outs[0], o)


@pytest.mark.slow
@pytest.mark.parametrize("n", [16384, 32768])
def test_config2_records_bit_identical(built, n):
    """n = 16384 (16 tiny + 3 zero columns) and n = 32768 (32 tiny + 6 zero
    columns, 8.6 GB): records equal the reference's, with no order-sensitive
    pivot decision; the residual is checked on the GPU (float64 products in
    torch)."""
    import delayed_pivoting as dp

    torch = _torch()
    name = f"config2_n{n}"
    if name not in gc.names():
        pytest.skip(f"{name} fixture not generated")
    a, case = gc.load(name)
    d = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    del a
    orig = d.clone()
    ipiv = np.zeros(n, dtype=np.int32)
    jpiv = np.zeros(n, dtype=np.int32)
    st, info = dp.delayed_getrf_cuda_device(n, n, d, n, ipiv, jpiv)
    torch.cuda.synchronize()
    assert st == 0 and info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])
    assert_no_near_ties(info)
    assert scaled_residual_gpu(torch, orig, d, n, info, ipiv, jpiv) <= 10.0
    del d, orig
    torch.cuda.empty_cache()


def scaled_residual_gpu(torch, orig_t, fac_t, n, info, ipiv, jpiv):
    """Square case: tensors are (n, n) holding the column-major matrix transposed."""
    F = fac_t.T  # column-major view -> actual matrix
    A = orig_t.T
    row = np.arange(n)
    col = np.arange(n)
    for k in range(info):
        row[[k, ipiv[k]]] = row[[ipiv[k], k]]
        col[[k, jpiv[k]]] = col[[jpiv[k], k]]
    PAQ = A[torch.from_numpy(row).cuda()][:, torch.from_numpy(col).cuda()]
    L = torch.tril(F, -1)
    L[:, info:] = 0
    L += torch.eye(n, dtype=F.dtype, device=F.device)
    U = torch.triu(F)
    U[info:, :] = 0
    U[info:, info:] = F[info:, info:]
    R = PAQ - L @ U
    return float(torch.linalg.norm(R) / (torch.linalg.norm(A) * n * 2.0**-53))


def _tie_matrix(kind):
    """300 x 300 N(0,1) with a planted decision at step 0: an exact tie
    (+10 / -10), a near-tie one ulp apart, or a clear gap; or, with column 0
    zero, an exact tie of the 2-D fallback search (+7 at column 4, -7 at
    column 2: the smaller column wins)."""
    import delayed_pivoting as dp

    a = dp.planted_matrix(300, 300, 606)
    a[:, 0] *= 0.1
    if kind == "exact":
        a[5, 0], a[9, 0] = 10.0, -10.0
    elif kind == "ulp":
        a[5, 0], a[9, 0] = 10.0, np.nextafter(10.0, 0.0)
    elif kind == "clear":
        a[5, 0], a[9, 0] = 10.0, 9.99
    else:  # fallback search tie
        a[:, 0] = 0.0
        a[:, 2:5] *= 0.1
        a[3, 4], a[6, 2] = 7.0, -7.0
    return a


@pytest.mark.parametrize("kind,flagged", [("exact", True), ("ulp", True), ("clear", False),
                                          ("fallback", True)])
def test_near_tie_detector_flags_planted_ties(built, kind, flagged):
    """The detector counts a planted tie (and only it); the decision itself
    still follows the reference's rule (first row; smaller column, then
    smaller row), so the records equal the oracle's."""
    import delayed_pivoting as dp
    import oracle as orc

    a = _tie_matrix(kind)
    o = a.copy(order="F")
    oi, oj, oinfo = orc.oracle_getrf(o)
    fac, ipiv, jpiv, info, st = run_device(a, 300, 300)
    assert st == 0 and info == oinfo
    np.testing.assert_array_equal(ipiv, oi)
    np.testing.assert_array_equal(jpiv, oj)
    rep = dp.getrf_last_report()
    assert rep["info"] == info and rep["decisions"] >= info
    if flagged:
        assert rep["near_ties"] >= 1, rep
        assert rep["max_closeness"] >= 1.0 - 2.0**-50, rep
    else:
        assert rep["near_ties"] == 0, rep
    if kind == "exact":
        assert ipiv[0] == 5
    if kind == "fallback":
        assert ipiv[0] == 6 and jpiv[0] == 2


def test_near_tie_report_of_failed_call(built):
    """A rejected call leaves a report with info = -1 and no decisions."""
    import delayed_pivoting as dp

    _torch()
    ipiv = np.zeros(4, dtype=np.int32)
    jpiv = np.zeros(4, dtype=np.int32)
    st, info = dp.delayed_getrf_cuda_device(4, 4, None, 4, ipiv, jpiv)
    assert st == dp.INVALID_ARGUMENT and info == -1
    rep = dp.getrf_last_report()
    assert rep["info"] == -1 and rep["decisions"] == 0 and rep["near_ties"] == 0


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (130, 70, 64), (1000, 3000, 256), (4099, 385, 100),
                                   (300, 20000, 32)])
@pytest.mark.parametrize("prec", ["x3", "x6"])
def test_mixed_schur_update_against_torch(built, M, N, K, prec):
    """The tensor-core update C -= A B (BF16 split, FP32 accumulation) against
    an FP64 torch product: |error| <= c K 2^-p max|A| max|B| with 2^-p the
    split's resolution (x3: 2^-16, x6: 2^-24, plus the FP32 accumulation);
    rows and columns outside C are untouched.  Many tiles per CTA (persistent
    grid) and ragged edges are covered."""
    import delayed_pivoting as dp

    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    lda, ldb, ldc = M + 3, K + 1, M + 5
    A = torch.randn(K, lda, dtype=torch.float64, device="cuda", generator=g)  # column-major lda x K
    B = torch.randn(N, ldb, dtype=torch.float64, device="cuda", generator=g)
    C = torch.randn(N, ldc, dtype=torch.float64, device="cuda", generator=g)
    C0 = C.clone()
    ref = C0[:, :M].T - A[:, :M].T @ B[:, :K].T
    p = dp.PRECISION_MIXED_BF16X3 if prec == "x3" else dp.PRECISION_MIXED_BF16X6
    assert dp.schur_update_mixed_device(M, N, K, A, lda, B, ldb, C, ldc, precision=p) == 0
    err = (C[:, :M].T - ref).abs().max().item()
    scale = A[:, :M].abs().max().item() * B[:, :K].abs().max().item()
    tol = K * scale * (2.0**-14 if prec == "x3" else 2.0**-21)
    assert err <= tol, (err, tol)
    assert torch.equal(C[:, M:], C0[:, M:])


def _nan_matrix(n, kind, seed):
    import delayed_pivoting as dp

    a = dp.planted_matrix(n, n, seed)
    if kind == "entry":
        a[n // 4, n // 3] = np.nan
    elif kind == "column":
        a[:, 10] = np.nan
    else:  # row
        a[n // 2, :] = np.nan
    return a


@pytest.mark.parametrize("n", [300, 700])
@pytest.mark.parametrize("kind", ["entry", "column", "row"])
def test_nan_inputs_follow_the_reference_gpu_rule(built, n, kind):
    """NaN never wins a pivot search (delayed_lu_cuda/delayed_dgetrf_cuda.cu:46):
    a NaN entry, a NaN column (delayed to the end) and a NaN row give the
    oracle's records and info on the single-CTA (n = 300) and the cluster
    panel (n = 700) paths, with no order-sensitive decision."""
    import oracle as orc

    a = _nan_matrix(n, kind, 31 + n)
    o = a.copy(order="F")
    oi, oj, oinfo = orc.oracle_getrf(o)
    fac, ipiv, jpiv, info, st = run_device(a, n, n)
    assert st == 0 and info == oinfo
    if kind != "entry":
        assert info == n - 1  # the NaN column / row ends as the delayed block
    np.testing.assert_array_equal(ipiv, oi)
    np.testing.assert_array_equal(jpiv, oj)
    assert_no_near_ties(info)


def test_autotuned_widths_keep_the_records(built, tmp_path):
    """dp_getrf_autotune picks a (panel width, outer block) pair for n's
    bucket; the default entry point then uses it and still reproduces the
    reference's records; the table survives a save / load round trip."""
    import delayed_pivoting as dp

    _torch()
    st, nb, nbo = dp.getrf_autotune(2000)
    assert st == 0 and nb in (32, 64, 128) and nbo in (64, 128, 256) and nb <= nbo
    a, case = gc.load("square_2000_zero20")
    fac, ipiv, jpiv, info, st = run_device(a, 2000, 2000)
    assert st == 0 and info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])
    assert_no_near_ties(info)
    path = tmp_path / "lu_tune.txt"
    assert dp.getrf_tune_save(path) == 0
    line = [ln.split() for ln in path.read_text().splitlines() if ln.split()[0] == "1024"]
    assert line == [["1024", "2047", str(nb), str(nbo)]]
    assert dp.getrf_tune_load(path) == 0
    bad = tmp_path / "bad.txt"
    bad.write_text("1000 2047 64 256\n")
    assert dp.getrf_tune_load(bad) == dp.INVALID_ARGUMENT
    # leave the process's table empty (later tests use the default widths)
    empty = tmp_path / "empty.txt"
    empty.write_text("")
    assert dp.getrf_tune_load(empty) == 0


@pytest.mark.parametrize("name", ["config1_n1024", "config1_n1024_column", "square_2000_zero20",
                                  "square_2000_zero20_column", "ref_far_pivot_70",
                                  "square_517_lda520", "tall_300x200", "wide_150x260"])
@pytest.mark.parametrize("kernel,rows,nb", [(1, 256, 64), (1, 512, 64), (1, 1024, 64),
                                            (1, 64, 13), (1, 700, 100), (3, 256, 64)])
def test_cluster_panels_keep_the_records(built, name, kernel, rows, nb):
    """Every panel of the factorisation on a cluster kernel: the register
    sub-panel one (panel_kernel 1) with 1, 2 and 4 rows per thread (rows per
    CTA up to 256, 512, 1024), odd widths and partial sub-panels, and the
    shared-memory one (panel_kernel 3): records equal the reference's, no
    order-sensitive decision, residual within the bound."""
    import oracle as orc

    a, case = gc.load(name)
    m, n = case["m"], case["n"]
    fac, ipiv, jpiv, info, st = run_device(a, m, n, nb=nb, panel_kernel=kernel, panel_rows=rows,
                                           policy=case["policy"])
    assert st == 0 and info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])
    assert_no_near_ties(info)
    assert orc.scaled_residual(a, fac, m, n, info, ipiv, jpiv) <= 10.0
