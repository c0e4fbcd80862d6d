"""Tests of the batched factorisation (dp_batch_*): thousands of small matrices
of uneven orders in one persistent launch, each with the single-matrix
semantics of delayed_lu/delayed_dgetrf.cpp:129-251.

CPU tests pin the oracle to the reference's records of a seeded 64-matrix
subset of the batched workload (tests/golden/batch/config4_subset64.npz,
written by tests/golden/make_golden.py from the reference's own CPU code) and
check the host-side argument handling.  GPU tests compare the batched kernel's
records bit for bit with that fixture and with the oracle, and its factors by
the scaled residual ||PAQ - LU||_F / (||A||_F n u) <= 10.

Inputs whose pivot decisions depend on rounding (an exactly dependent column,
whose Schur complement is rounding noise) are not used: records are only
comparable where every decision has a clear winner."""
from pathlib import Path

import numpy as np
import pytest

FIXTURE = Path(__file__).resolve().parent / "golden" / "batch" / "config4_subset64.npz"


def fixture():
    with np.load(FIXTURE) as z:
        return {k: z[k] for k in z.files}


def split_records(flat, ns):
    out, pos = [], 0
    for n in ns:
        out.append(flat[pos:pos + int(n)])
        pos += int(n)
    return out


# ---------------------------------------------------------------- CPU ----

def test_fixture_recipe_is_stable():
    import delayed_pivoting as dp

    f = fixture()
    ns, nz = dp.batch_orders(int(f["count"]), int(f["seed"]))
    assert np.array_equal(ns, f["ns"]) and np.array_equal(nz, f["n_zero"])
    assert ns.min() >= 32 and ns.max() <= 512
    # the subset exercises delays and fallbacks
    assert (f["info"] < ns).sum() >= 10


def test_oracle_matches_reference_batch_records(built):
    import delayed_pivoting as dp
    import oracle as orc

    f = fixture()
    ns, nz, seed = f["ns"], f["n_zero"], int(f["seed"])
    ip = split_records(f["ipiv"], ns)
    jp = split_records(f["jpiv"], ns)
    for i in range(0, len(ns), 4):  # every 4th matrix keeps the CPU suite short
        a = dp.batch_matrix(ns, nz, seed, i)
        n = int(ns[i])
        ipiv, jpiv, info = orc.oracle_getrf(a, n, n, nb=16)
        assert info == f["info"][i], i
        assert np.array_equal(ipiv, ip[i]) and np.array_equal(jpiv, jp[i]), i


def test_batch_create_rejects_bad_arguments(built):
    import delayed_pivoting as dp

    for ns in ([0], [513], [5, -1]):
        with pytest.raises(dp.BatchError) as e:
            dp.Batch(ns)
        assert e.value.status == dp.INVALID_ARGUMENT
    for nb in (0, 33):
        with pytest.raises(dp.BatchError) as e:
            dp.Batch([8], options=dp.batch_options(nb_bucket=nb))
        assert e.value.status == dp.INVALID_ARGUMENT
    with pytest.raises(dp.BatchError):
        dp.Batch([8], options=dp.batch_options(threshold=-1.0))
    with pytest.raises(dp.BatchError):
        dp.Batch([8], offsets=[-4])


def test_tune_table_round_trip(tmp_path):
    import delayed_pivoting as dp

    opt = dp.batch_options(nb_bucket=[8, 12, 24, 32])
    path = tmp_path / "tune.txt"
    assert dp.batch_tune_save(path, opt) == 0
    lines = path.read_text().split("\n")
    assert lines[0].split() == ["1", "63", "8"] and lines[3].split() == ["256", "512", "32"]
    st, back = dp.batch_tune_load(path)
    assert st == 0 and list(back.nb_bucket) == [8, 12, 24, 32]
    path.write_text("1 63 8\n64 127 99\n")
    assert dp.batch_tune_load(path)[0] == dp.INVALID_ARGUMENT


# ---------------------------------------------------------------- GPU ----

def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def run_batch(ns, n_zero, seed, options=None, graph=False, offsets=None, matrices=None):
    """Factors a batch on the GPU; returns (batch, host buffer before, factors
    after, ipiv, jpiv, info)."""
    import delayed_pivoting as dp

    torch = _torch()
    b = dp.Batch(ns, offsets=offsets, options=options)
    host = np.zeros(max(b.total_elements, 1), dtype=np.float64)
    if matrices is None:
        dp.fill_batch(host, b.offsets, ns, n_zero, seed)
    else:
        for off, a in zip(b.offsets, matrices):
            host[off:off + a.size] = a.ravel(order="F")
    d = torch.from_numpy(host).cuda()
    rec = max(b.total_records, 1)
    d_ipiv = torch.full((rec,), -7, dtype=torch.int32, device="cuda")
    d_jpiv = torch.full((rec,), -7, dtype=torch.int32, device="cuda")
    d_info = torch.full((max(len(ns), 1),), -7, dtype=torch.int32, device="cuda")
    fn = b.getrf_graph if graph else b.getrf_async
    assert fn(d, d_ipiv, d_jpiv, d_info) == 0
    torch.cuda.synchronize()
    return (b, host, d.cpu().numpy(), d_ipiv.cpu().numpy(), d_jpiv.cpu().numpy(),
            d_info.cpu().numpy())


def matrix_at(buf, off, n):
    return np.asfortranarray(buf[off:off + n * n].reshape(n, n, order="F"))


def check_residuals(b, host, fac, ns, ipiv, jpiv, info, every=1):
    import oracle as orc

    ip = split_records(ipiv, ns)
    jp = split_records(jpiv, ns)
    worst = 0.0
    for i in range(0, len(ns), every):
        n = int(ns[i])
        a = matrix_at(host, b.offsets[i], n)
        f = matrix_at(fac, b.offsets[i], n)
        r = orc.scaled_residual(a, f, n, n, int(info[i]), ip[i], jp[i])
        worst = max(worst, r)
        assert r <= 10.0, (i, n, r)
    return worst


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_batched_records_equal_reference_subset(built, graph):
    f = fixture()
    ns, nz, seed = f["ns"], f["n_zero"], int(f["seed"])
    b, host, fac, ipiv, jpiv, info = run_batch(ns, nz, seed, graph=graph)
    assert np.array_equal(info, f["info"])
    assert np.array_equal(ipiv, f["ipiv"])
    assert np.array_equal(jpiv, f["jpiv"])
    # no pivot decision of the launch was order-sensitive (near-tie detector)
    rep = b.last_report()
    assert rep["near_ties"] == 0 and rep["decisions"] >= int(info.sum()), rep
    assert rep["info"] == len(ns)
    check_residuals(b, host, fac, ns, ipiv, jpiv, info)


@pytest.mark.gpu
@pytest.mark.parametrize("nb", [1, 5, 8, 13, 16, 24, 32])
def test_batched_panel_width_does_not_change_records(built, nb):
    import delayed_pivoting as dp

    f = fixture()
    ns, nz, seed = f["ns"], f["n_zero"], int(f["seed"])
    b, host, fac, ipiv, jpiv, info = run_batch(ns, nz, seed,
                                               options=dp.batch_options(nb_bucket=nb))
    assert np.array_equal(info, f["info"])
    assert np.array_equal(ipiv, f["ipiv"]) and np.array_equal(jpiv, f["jpiv"])
    assert b.last_report()["near_ties"] == 0
    check_residuals(b, host, fac, ns, ipiv, jpiv, info, every=3)


@pytest.mark.gpu
def test_batched_graph_replay_is_bitwise_repeatable(built):
    import delayed_pivoting as dp

    torch = _torch()
    ns, nz = dp.batch_orders(300, 77)
    b = dp.Batch(ns)
    host = np.zeros(b.total_elements, dtype=np.float64)
    dp.fill_batch(host, b.offsets, ns, nz, 77)
    src = torch.from_numpy(host).cuda()
    outs = []
    for graph in (False, True, True):
        d = src.clone()
        ip = torch.empty(b.total_records, dtype=torch.int32, device="cuda")
        jp = torch.empty_like(ip)
        inf = torch.empty(len(ns), dtype=torch.int32, device="cuda")
        fn = b.getrf_graph if graph else b.getrf_async
        assert fn(d, ip, jp, inf) == 0
        torch.cuda.synchronize()
        outs.append((d.cpu().numpy(), ip.cpu().numpy(), jp.cpu().numpy(), inf.cpu().numpy()))
    for o in outs[1:]:
        for x, y in zip(outs[0], o):
            assert np.array_equal(x, y)


@pytest.mark.gpu
def test_batched_matches_oracle_and_single_matrix_path(built):
    """A fresh seeded batch: records equal the oracle's and the single-matrix
    GPU path's for every matrix."""
    import delayed_pivoting as dp
    import oracle as orc

    torch = _torch()
    ns, nz = dp.batch_orders(96, 4242)
    b, host, fac, ipiv, jpiv, info = run_batch(ns, nz, 4242)
    ip = split_records(ipiv, ns)
    jp = split_records(jpiv, ns)
    for i in range(len(ns)):
        n = int(ns[i])
        a = matrix_at(host, b.offsets[i], n)
        o_ip, o_jp, o_info = orc.oracle_getrf(a.copy(order="F"), n, n, nb=32)
        assert info[i] == o_info and np.array_equal(ip[i], o_ip) and np.array_equal(jp[i], o_jp)
        if i % 8 == 0:
            d = torch.from_numpy(a.T.copy()).cuda()
            s_ip = np.zeros(n, dtype=np.int32)
            s_jp = np.zeros(n, dtype=np.int32)
            st, s_info = dp.delayed_getrf_cuda_device(n, n, d, n, s_ip, s_jp)
            assert st == 0 and s_info == info[i]
            assert np.array_equal(s_ip, ip[i]) and np.array_equal(s_jp, jp[i])
    check_residuals(b, host, fac, ns, ipiv, jpiv, info, every=2)


@pytest.mark.gpu
def test_batched_threshold_matches_oracle(built):
    """threshold > 0: planted 1e-18 columns become fallbacks / delays."""
    import delayed_pivoting as dp
    import oracle as orc

    mats = [dp.planted_matrix(n, n, 900 + n, n_tiny=t, n_zero=z)
            for n, t, z in [(40, 2, 0), (100, 3, 1), (200, 4, 2), (333, 5, 0), (512, 6, 1)]]
    ns = np.array([a.shape[0] for a in mats], dtype=np.int32)
    for thr in (1e-12, 1e-3):
        b, host, fac, ipiv, jpiv, info = run_batch(
            ns, None, 0, options=dp.batch_options(threshold=thr), matrices=mats)
        ip = split_records(ipiv, ns)
        jp = split_records(jpiv, ns)
        for i, a in enumerate(mats):
            n = int(ns[i])
            o_ip, o_jp, o_info = orc.oracle_getrf(a.copy(order="F"), n, n, nb=32, threshold=thr)
            assert info[i] == o_info, (thr, n)
            assert np.array_equal(ip[i], o_ip) and np.array_equal(jp[i], o_jp), (thr, n)


@pytest.mark.gpu
def test_batched_edge_cases(built):
    import delayed_pivoting as dp
    import oracle as orc

    rng = np.random.default_rng(5)
    mats = []
    mats.append(np.zeros((1, 1), order="F"))                      # info 0
    mats.append(np.full((1, 1), -3.0, order="F"))                 # info 1
    mats.append(np.asfortranarray([[0.0, 2.0], [1.0, 0.0]]))      # pivot from row 1
    mats.append(np.zeros((9, 9), order="F"))                      # all zero: info 0
    a = np.asfortranarray(rng.standard_normal((70, 70)))
    a[:, 0] = 0.0                                                  # fallback at step 0
    mats.append(a)
    a = np.asfortranarray(rng.standard_normal((130, 130)))
    a[:, 5] = 0.0                                                  # fallbacks mid-panel
    a[:, 37] = 0.0
    a[:3, 60] = 0.0                                                # zero head of a column
    mats.append(a)
    a = np.asfortranarray(rng.standard_normal((512, 512)))
    a[:, [7, 200, 511]] = 0.0                                      # largest order
    mats.append(a)
    e = np.asfortranarray(np.diag(rng.uniform(1, 2, 33)))
    e[[0, 1]] = e[[1, 0]]                                          # zero ties below pivots
    mats.append(e)
    ns = np.array([m.shape[0] for m in mats], dtype=np.int32)
    # explicit offsets with gaps, matrices stored in reverse order
    offs, pos = [], 1000
    for m in mats[::-1]:
        offs.append(pos)
        pos += m.size + 37
    offs = offs[::-1]
    b, host, fac, ipiv, jpiv, info = run_batch(ns, None, 0, offsets=offs, matrices=mats)
    ip = split_records(ipiv, ns)
    jp = split_records(jpiv, ns)
    for i, m in enumerate(mats):
        n = int(ns[i])
        o_ip, o_jp, o_info = orc.oracle_getrf(m.copy(order="F"), n, n, nb=32)
        assert info[i] == o_info, i
        assert np.array_equal(ip[i], o_ip) and np.array_equal(jp[i], o_jp), i
    assert list(info[:4]) == [0, 1, 2, 0]
    check_residuals(b, host, fac, ns, ipiv, jpiv, info)
    # gaps between matrices are untouched
    mask = np.ones(b.total_elements, dtype=bool)
    for off, m in zip(offs, mats):
        mask[off:off + m.size] = False
    assert np.array_equal(fac[mask], host[mask])


@pytest.mark.gpu
def test_batched_autotune_fills_every_bucket(built, tmp_path):
    import delayed_pivoting as dp

    _torch()
    st, opt = dp.batch_autotune(samples=4)
    assert st == 0
    assert all(1 <= v <= dp.BATCH_MAX_NB for v in opt.nb_bucket)
    assert dp.batch_tune_save(tmp_path / "t.txt", opt) == 0
    # the tuned widths keep the records
    f = fixture()
    ns, nz, seed = f["ns"], f["n_zero"], int(f["seed"])
    _, _, _, ipiv, jpiv, info = run_batch(ns, nz, seed, options=opt)
    assert np.array_equal(info, f["info"]) and np.array_equal(ipiv, f["ipiv"])


@pytest.mark.gpu
def test_batched_empty_batch(built):
    import delayed_pivoting as dp

    torch = _torch()
    b = dp.Batch([])
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    i = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert b.getrf_async(x, i, i, i) == 0
    assert b.getrf_graph(x, i, i, i) == 0


@pytest.mark.gpu
def test_batched_near_tie_detector_counts_planted_ties(built):
    """Two matrices of one launch carry a planted exact tie (step 0 column
    search; 2-D fallback search), one does not: the launch's report counts
    the two ties, and the records still follow the reference's tie rule."""
    import delayed_pivoting as dp
    import oracle as orc

    mats = []
    for seed, kind in ((11, "col"), (12, "none"), (13, "fallback")):
        a = dp.planted_matrix(200, 200, seed)
        a[:, 0] *= 0.1
        if kind == "col":
            a[5, 0], a[9, 0] = 10.0, -10.0
        elif kind == "fallback":
            a[:, 0] = 0.0
            a[:, 2:5] *= 0.1
            a[3, 4], a[6, 2] = 7.0, -7.0
        mats.append(a)
    ns = np.array([200, 200, 200], dtype=np.int32)
    b, host, fac, ipiv, jpiv, info = run_batch(ns, None, 0, matrices=mats)
    ip, jp = split_records(ipiv, ns), split_records(jpiv, ns)
    for i, a in enumerate(mats):
        oi, oj, oinfo = orc.oracle_getrf(a.copy(order="F"))
        assert info[i] == oinfo
        assert np.array_equal(ip[i], oi) and np.array_equal(jp[i], oj)
    rep = b.last_report()
    assert rep["near_ties"] == 2, rep
    assert rep["max_closeness"] == 1.0 and rep["info"] == 3


@pytest.mark.gpu
def test_batched_nan_inputs_follow_the_reference_gpu_rule(built):
    """NaN never wins in the batched kernel either: NaN entry / column / row
    matrices get the oracle's records."""
    import delayed_pivoting as dp
    import oracle as orc

    mats = []
    for seed, kind in ((41, "entry"), (42, "column"), (43, "row")):
        a = dp.planted_matrix(250, 250, seed)
        if kind == "entry":
            a[60, 80] = np.nan
        elif kind == "column":
            a[:, 10] = np.nan
        else:
            a[125, :] = np.nan
        mats.append(a)
    ns = np.array([250, 250, 250], dtype=np.int32)
    b, host, fac, ipiv, jpiv, info = run_batch(ns, None, 0, matrices=mats)
    ip, jp = split_records(ipiv, ns), split_records(jpiv, ns)
    for i, a in enumerate(mats):
        oi, oj, oinfo = orc.oracle_getrf(a.copy(order="F"))
        assert info[i] == oinfo
        assert np.array_equal(ip[i], oi) and np.array_equal(jp[i], oj)
    assert b.last_report()["near_ties"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision,bound", [(1, 3e-3), (2, 1e-5)])
def test_batched_mixed_forms(built, precision, bound):
    """The mixed forms of the batched launch (BF16 split trailing updates,
    3 or 6 products with FP32 accumulation; panels, solves and pivot decisions
    in FP64): relative residual ||PAQ - LU|| / ||A|| at the level of the
    update's rounding, the same delays as the FP64 form (exact zero columns
    stay exactly zero), graph replay bitwise equal to the direct launch, and
    FP64 refinement with the mixed factors reaching 1e-14 on a well-conditioned
    matrix."""
    import delayed_pivoting as dp
    import oracle as orc

    torch = _torch()
    ns, nz = dp.batch_orders(200, 5150)
    opt = dp.batch_options(precision=precision)
    b64, host, fac64, ip64, jp64, info64 = run_batch(ns, nz, 5150)
    b, host2, fac, ipiv, jpiv, info = run_batch(ns, nz, 5150, options=opt)
    assert np.array_equal(host, host2)
    assert np.array_equal(info, info64)
    _, _, facg, ipg, jpg, infog = run_batch(ns, nz, 5150, options=opt, graph=True)
    assert np.array_equal(fac, facg) and np.array_equal(ipiv, ipg) and np.array_equal(info, infog)
    ip = split_records(ipiv, ns)
    jp = split_records(jpiv, ns)
    worst = 0.0
    for i in range(len(ns)):
        n = int(ns[i])
        a = matrix_at(host, b.offsets[i], n)
        f = matrix_at(fac, b.offsets[i], n)
        r, an = orc.residual(a, f, n, n, int(info[i]), ip[i], jp[i])
        worst = max(worst, r / an)
    assert worst <= bound, worst
    # FP64 refinement with the mixed factors of a full-rank matrix
    i = int(np.argmax(np.where(info == ns, ns, 0)))
    n = int(ns[i])
    a = matrix_at(host, b.offsets[i], n)
    f = matrix_at(fac, b.offsets[i], n)
    L = np.tril(f, -1) + np.eye(n)
    U = np.triu(f)

    def solve(rhs):
        x = rhs.copy()
        for k in range(n):  # P: the row swaps in step order
            x[[k, ip[i][k]]] = x[[ip[i][k], k]]
        x = np.linalg.solve(U, np.linalg.solve(L, x))
        for k in range(n - 1, -1, -1):  # Q: the column swaps undone in reverse
            x[[k, jp[i][k]]] = x[[jp[i][k], k]]
        return x

    rng = np.random.default_rng(7)
    xt = rng.standard_normal(n)
    rhs = a @ xt
    x = solve(rhs)
    for _ in range(10):
        r = rhs - a @ x
        if np.abs(r).max() / (np.abs(a).max() * np.abs(x).max() * n) <= 1e-16:
            break
        x = x + solve(r)
    berr = np.abs(rhs - a @ x).max() / (np.abs(a).sum(axis=1).max() * np.abs(x).max() + np.abs(rhs).max())
    assert berr <= 1e-14, berr
