"""CPU tests of the oracle: the plain-C restatement of the reference's
delayed_getrf is pinned against golden records produced by the reference's
own CPU code (tests/golden/*.npz) and, when the reference build is present,
against that build directly on fresh seeded inputs."""
import numpy as np
import pytest

import golden_cases as gc


def test_mt19937_64_engine_matches_std(built):
    import delayed_pivoting as dp

    # C++ [rand.predef]: the 10000th output of a default-constructed
    # std::mt19937_64 (seed 5489) is 9981545732273789042.
    assert dp.mt64_nth(5489, 10000) == 9981545732273789042


def test_generator_is_deterministic(built):
    import delayed_pivoting as dp

    a = dp.planted_matrix(64, 48, 99, 2, 3, lda=70)
    b = dp.planted_matrix(64, 48, 99, 2, 3, lda=70)
    assert np.array_equal(a, b)
    assert np.all(a[64:, :] == 0.0)
    zero_cols = np.where(np.all(a[:64] == 0.0, axis=0))[0]
    assert len(zero_cols) == 3
    tiny = np.where((np.abs(a[:64]).max(axis=0) < 1e-16) & (np.abs(a[:64]).max(axis=0) > 0))[0]
    assert len(tiny) == 2


@pytest.mark.parametrize("name", gc.names(max_elems=4096 * 4096))
def test_oracle_matches_golden(built, name):
    import oracle as orc

    a, case = gc.load(name)
    m, n = case["m"], case["n"]
    f = a.copy(order="F")
    ipiv, jpiv, info = orc.oracle_getrf(f, m, n, policy=case["policy"])
    assert info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])
    if m * n <= 2100 * 2100:
        assert orc.scaled_residual(a, f, m, n, info, ipiv, jpiv) <= 10.0


@pytest.mark.parametrize("name", gc.names(max_elems=2100 * 2100))
def test_reference_build_reproduces_golden(built, name):
    import oracle as orc

    if not orc.ref_available():
        pytest.skip("reference CPU build not present")
    a, case = gc.load(name)
    f = a.copy(order="F")
    fn = orc.ref_getrf if case["policy"] == 0 else orc.ref_getrf_column
    ipiv, jpiv, info = fn(f, case["m"], case["n"])
    assert info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])


@pytest.mark.parametrize("nb", [1, 3, 16, 64, 200])
def test_panel_width_does_not_change_records(built, nb):
    import oracle as orc

    a, case = gc.load("config1_n1024")
    ipiv, jpiv, info = orc.oracle_getrf(a.copy(order="F"), nb=nb)
    assert info == case["info"]
    np.testing.assert_array_equal(ipiv, case["ipiv"])
    np.testing.assert_array_equal(jpiv, case["jpiv"])


@pytest.mark.parametrize("seed", range(12))
def test_oracle_matches_reference_on_random_shapes(built, seed):
    import delayed_pivoting as dp
    import oracle as orc

    if not orc.ref_available():
        pytest.skip("reference CPU build not present")
    rng = np.random.default_rng(seed)
    m = int(rng.integers(1, 300))
    n = int(rng.integers(1, 300))
    lda = m + int(rng.integers(0, 5))
    nz = int(rng.integers(0, max(1, min(m, n) // 4) + 1))
    nt = int(rng.integers(0, 3)) if n - nz > 2 else 0
    nz = min(nz, n - nt)
    a = dp.planted_matrix(m, n, 1000 + seed, nt, nz, lda=lda)
    for policy in (0, 1):
        r = a.copy(order="F")
        o = a.copy(order="F")
        fn = orc.ref_getrf if policy == 0 else orc.ref_getrf_column
        ri, rj, rinfo = fn(r, m, n)
        oi, oj, oinfo = orc.oracle_getrf(o, m, n, nb=int(rng.integers(1, 100)), policy=policy)
        assert rinfo == oinfo
        np.testing.assert_array_equal(ri, oi)
        np.testing.assert_array_equal(rj, oj)
        assert orc.scaled_residual(a, o, m, n, oinfo, oi, oj) <= 10.0


def test_threshold_extension_delays_tiny_columns(built):
    """threshold > 0: tiny (1e-18) columns are pushed into the delayed suffix;
    the delayed block then holds nothing above the threshold."""
    import oracle as orc

    a, case = gc.load("config1_n1024")
    f = a.copy(order="F")
    thr = 1e-12
    ipiv, jpiv, info = orc.oracle_getrf(f, threshold=thr)
    assert info == 1024 - 16 - 4
    assert np.abs(f[info:, info:]).max() <= thr
    assert orc.scaled_residual(a, f, 1024, 1024, info, ipiv, jpiv) <= 10.0
    # threshold 0 is the reference exactly
    ipiv0, jpiv0, info0 = orc.oracle_getrf(a.copy(order="F"), threshold=0.0)
    np.testing.assert_array_equal(ipiv0, case["ipiv"])
    assert info0 == case["info"]


def test_oracle_rejects_invalid_arguments(built):
    import oracle as orc

    a = np.zeros((4, 4), order="F")
    assert orc.oracle_getrf(a, 5, 4)[2] == -1  # lda < m
    assert orc.oracle_getrf(a, -1, 4)[2] == -1
    assert orc.oracle_getrf(a, 4, 4, nb=0)[2] == -1
    assert orc.oracle_getrf(a, 4, 4, threshold=-1.0)[2] == -1


def test_empty_matrix(built):
    import oracle as orc

    a = np.zeros((1, 1), order="F")
    _, _, info = orc.oracle_getrf(a, 0, 0)
    assert info == 0


@pytest.mark.parametrize("seed", range(10))
def test_oracle_matches_reference_on_exact_ties_and_rank_deficiency(built, seed):
    """Small-integer matrices: eliminations stay exact, so columns tie in
    magnitude (the first row wins, delayed_dgetrf.cpp:164-176 through idamax)
    and become exactly zero part-way (the full-pivot fallback and the delayed
    suffix, :183-218); duplicated columns force rank deficiency."""
    import oracle as orc

    if not orc.ref_available():
        pytest.skip("reference CPU build not present")
    rng = np.random.default_rng(500 + seed)
    m = int(rng.integers(2, 40))
    n = int(rng.integers(2, 40))
    a = np.asfortranarray(rng.integers(-2, 3, size=(m, n)).astype(np.float64))
    for _ in range(int(rng.integers(0, 3))):  # duplicated columns
        a[:, int(rng.integers(0, n))] = a[:, int(rng.integers(0, n))]
    for policy in (0, 1):
        r = a.copy(order="F")
        o = a.copy(order="F")
        fn = orc.ref_getrf if policy == 0 else orc.ref_getrf_column
        ri, rj, rinfo = fn(r, m, n)
        oi, oj, oinfo = orc.oracle_getrf(o, m, n, policy=policy)  # the reference's nb = 64
        assert rinfo == oinfo
        np.testing.assert_array_equal(ri, oi)
        np.testing.assert_array_equal(rj, oj)
