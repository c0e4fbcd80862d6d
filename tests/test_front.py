"""Multifrontal hand-off: partial factorisation of a front whose leading p
rows / columns are fully summed (dp_front_factor) and extend-add of its
contribution block into a parent front (dp_extend_add).

The reference has no code for this path (its design document describes it,
doc/...LU方法.md:228-457), so the checks are: the NumPy/C restatement
(oracle.oracle_front) against the Schur-complement identity on CPU, and the
device result against the restatement - records bit-equal (the fully-summed
block is the reference's delayed_getrf), factors and contribution block to
rounding."""
import numpy as np
import pytest

import oracle as orc


def make_front(m, n, p, seed, zero_tail=0, zero_col=None):
    """A seeded front; the last `zero_tail` rows and columns of the fully-
    summed block are zero there (they can only be delayed), `zero_col` a
    column that is zero inside the fully-summed rows only (a fallback)."""
    rng = np.random.default_rng(seed)
    f = np.asfortranarray(rng.standard_normal((m, n)))
    if zero_tail:
        f[p - zero_tail:p, :p] = 0.0
        f[:p, p - zero_tail:p] = 0.0
    if zero_col is not None:
        f[:p, zero_col] = 0.0
    return f


def permuted(f, p, ipiv, jpiv):
    g = np.array(f, copy=True)
    g[:p, :] = g[orc._composite(ipiv, p), :]
    g[:, :p] = g[:, orc._composite(jpiv, p)]
    return g


CASES = [(120, 110, 50, 1, 0, None), (96, 96, 40, 2, 3, None), (80, 140, 64, 3, 0, 5),
         (200, 150, 100, 4, 4, 17), (64, 64, 64, 5, 0, None), (70, 90, 0, 6, 0, None)]


@pytest.mark.parametrize("m,n,p,seed,tail,zc", CASES)
def test_oracle_front_contribution_block_is_the_schur_complement(m, n, p, seed, tail, zc):
    f = make_front(m, n, p, seed, tail, zc)
    k, ipiv, jpiv, out = orc.oracle_front(f, p)
    assert 0 <= k <= p
    if tail:
        assert k <= p - tail  # the zero tail can only be delayed
    g = permuted(f, p, ipiv, jpiv)
    # L (first k columns) U (first k rows) + [0 0; 0 S] reproduces the permuted front
    L = np.tril(out[:, :k], -1) + np.eye(m, k)
    U = np.triu(out[:k, :])
    rec = L @ U
    rec[k:, k:] += out[k:, k:]
    assert np.abs(rec - g).max() <= 1e-11 * max(1.0, np.abs(g).max())
    if k:
        s = g[k:, k:] - g[k:, :k] @ np.linalg.solve(g[:k, :k], g[:k, k:])
        assert np.allclose(out[k:, k:], s, rtol=1e-9, atol=1e-10)


# ---------------------------------------------------------------- GPU ----

def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,p,seed,tail,zc", CASES + [(1500, 1400, 700, 7, 5, 300)])
def test_front_factor_matches_restatement(built, m, n, p, seed, tail, zc):
    import delayed_pivoting as dp

    torch = _torch()
    f = make_front(m, n, p, seed, tail, zc)
    k0, ip0, jp0, out0 = orc.oracle_front(f, p)
    d = torch.from_numpy(np.ascontiguousarray(f.T)).cuda()
    rows = np.arange(1000, 1000 + m, dtype=np.int32)
    cols = np.arange(5000, 5000 + n, dtype=np.int32)
    st, k, ipiv, jpiv = dp.front_factor(m, n, p, d, m, rows, cols)
    torch.cuda.synchronize()
    assert st == dp.SUCCESS and k == k0
    np.testing.assert_array_equal(ipiv, ip0)
    np.testing.assert_array_equal(jpiv, jp0)
    out = np.asfortranarray(d.cpu().numpy().T)
    scale = max(1.0, float(np.abs(out0).max()))
    assert np.abs(out - out0).max() <= 1e-10 * scale * max(m, n) ** 0.5
    np.testing.assert_array_equal(rows[:p], 1000 + orc._composite(ip0, p))
    np.testing.assert_array_equal(cols[:p], 5000 + orc._composite(jp0, p))
    np.testing.assert_array_equal(rows[p:], np.arange(1000 + p, 1000 + m))


@pytest.mark.gpu
def test_front_factor_rejects_bad_arguments(built):
    import delayed_pivoting as dp

    _torch()
    assert dp.front_factor(10, 10, 11, 0x1000, 10)[0] == dp.INVALID_ARGUMENT
    assert dp.front_factor(10, 10, 5, 0x1000, 9)[0] == dp.INVALID_ARGUMENT
    assert dp.front_factor(10, 10, -1, 0x1000, 10)[0] == dp.INVALID_ARGUMENT


@pytest.mark.gpu
def test_extend_add_into_parent(built):
    """A child's contribution block, factored by dp_front_factor, scattered
    into its parent through the global index lists; a second child adds to
    overlapping rows in stream order."""
    import delayed_pivoting as dp

    torch = _torch()
    rng = np.random.default_rng(11)
    parent_idx = np.sort(rng.choice(5000, 300, replace=False)).astype(np.int32)
    P = np.asfortranarray(rng.standard_normal((300, 300)))
    dP = torch.from_numpy(np.ascontiguousarray(P.T)).cuda()
    expect = P.copy()
    for child, (m, p) in enumerate(((180, 60), (150, 40))):
        f = make_front(m, m, p, 20 + child)
        # the child's non-fully-summed indices all belong to the parent
        rows = np.concatenate([np.arange(9000 + 100 * child, 9000 + 100 * child + p),
                               rng.choice(parent_idx, m - p, replace=False)]).astype(np.int32)
        cols = rows.copy()
        d = torch.from_numpy(np.ascontiguousarray(f.T)).cuda()
        st, k, _, _ = dp.front_factor(m, m, p, d, m, rows, cols)
        assert st == dp.SUCCESS and k == p
        out = d.cpu().numpy().T
        cb = np.asfortranarray(out[k:, k:])
        pos_r = np.searchsorted(parent_idx, rows[k:]).astype(np.int32)
        pos_c = np.searchsorted(parent_idx, cols[k:]).astype(np.int32)
        assert np.array_equal(parent_idx[pos_r], rows[k:])
        d_cb = d.T[k:, k:].T  # the block in place: column-major, leading dimension m
        assert dp.extend_add(m - k, m - k, d_cb.data_ptr(), m, torch.from_numpy(pos_r).cuda(),
                             torch.from_numpy(pos_c).cuda(), dP, 300) == dp.SUCCESS
        expect[np.ix_(pos_r, pos_c)] += cb
    torch.cuda.synchronize()
    got = dP.cpu().numpy().T
    assert np.abs(got - expect).max() <= 1e-13 * np.abs(expect).max()


def test_bench_front_flops_and_reference_arm():
    """bench.py --workload front: the partial-LU flop count matches the exact
    sum over the eliminated pivots to leading order, and the reference arm
    reports that the reference has no code for the hand-off."""
    import importlib.util
    import json
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    spec = importlib.util.spec_from_file_location("bench_mod", root / "bench.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    for m, n, k in ((400, 400, 200), (1000, 800, 300)):
        exact = sum(2 * (m - j - 1) * (n - j - 1) for j in range(k))
        assert abs(b.front_flops(m, n, k) / exact - 1.0) < 0.01
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference",
                        "--workload", "front"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line
