"""GPU tests of the solve layer: getrs with the swap-history factors, and the
mixed-precision LU + FP64 iterative refinement (dp_gesv_ir_device).

getrs is checked on an explicit factorisation P*A*Q = L*U built on the CPU
with random row and column swap histories (a nonsingular matrix never needs a
column fallback at threshold 0, so this is how the Q path is exercised).
Refinement is checked on A = U diag(sigma) V^T with geometric singular values
(kappa = 1e2 .. 1e10): normwise backward error <= 1e-14 and forward error
within kappa * 1e-14; kappa = 1e10 must fall back to the FP64 factorisation.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def colmajor(torch, a):
    """Host Fortran array -> device tensor holding the column-major matrix."""
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def from_dev(t):
    return np.asfortranarray(t.cpu().numpy().T)


@pytest.mark.parametrize("n,nrhs", [(1, 1), (7, 3), (130, 1), (300, 5), (1000, 64)])
def test_getrs_with_row_and_column_histories(n, nrhs):
    import delayed_pivoting as dp

    torch = _torch()
    rng = np.random.default_rng(n + nrhs)
    L = np.tril(rng.standard_normal((n, n)) * 0.1, -1) + np.eye(n)
    U = np.triu(rng.standard_normal((n, n)) * 0.1, 1) + np.diag(rng.uniform(1.0, 2.0, n))
    ipiv = np.array([rng.integers(k, n) for k in range(n)], dtype=np.int32)
    jpiv = np.array([rng.integers(k, n) for k in range(n)], dtype=np.int32)
    lu = np.tril(L, -1) + U
    # P A Q = L U  ->  A = P^T (L U) Q^T with P, Q the replayed swap histories
    row = np.arange(n)
    col = np.arange(n)
    for k in range(n):
        row[[k, ipiv[k]]] = row[[ipiv[k], k]]
        col[[k, jpiv[k]]] = col[[jpiv[k], k]]
    PAQ = L @ U
    A = np.empty_like(PAQ)
    A[np.ix_(row, col)] = PAQ
    x_true = rng.standard_normal((n, nrhs))
    b = A @ x_true
    d_lu = colmajor(torch, np.asfortranarray(lu))
    d_b = colmajor(torch, np.asfortranarray(b))
    st = dp.getrs_device(n, nrhs, d_lu, n, ipiv, jpiv, d_b, n)
    assert st == 0
    x = from_dev(d_b)
    np.testing.assert_allclose(x, x_true, rtol=1e-9, atol=1e-9)


def test_getrs_rejects_bad_histories():
    import delayed_pivoting as dp

    torch = _torch()
    d = torch.zeros(4, 4, dtype=torch.float64, device="cuda")
    b = torch.zeros(1, 4, dtype=torch.float64, device="cuda")
    bad = np.array([0, 0, 2, 3], dtype=np.int32)  # ipiv[1] < 1
    ok = np.arange(4, dtype=np.int32)
    assert dp.getrs_device(4, 1, d, 4, bad, ok, b, 4) == dp.INVALID_ARGUMENT
    assert dp.getrs_device(4, 1, d, 3, ok, ok, b, 4) == dp.INVALID_ARGUMENT


def devcopy(t):
    """Column-major device copy of a (rows x cols) tensor.  `.T.contiguous()`
    alone aliases the input when one dimension is 1."""
    return t.T.contiguous().clone()


def conditioned(torch, n, kappa, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    u, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    v, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    sigma = torch.logspace(0, -np.log10(kappa), n, dtype=torch.float64, device="cuda")
    return (u * sigma) @ v.T, g


@pytest.mark.parametrize("kappa", [1e2, 1e4, 1e6, 1e10])
@pytest.mark.parametrize("nrhs", [1, 64])
@pytest.mark.parametrize("precision", [1, 2])  # BF16x3, BF16x6
def test_mixed_ir_reaches_fp64_backward_error(kappa, nrhs, precision):
    import delayed_pivoting as dp

    torch = _torch()
    n = 768
    A, g = conditioned(torch, n, kappa, seed=int(np.log10(kappa)) * 10 + nrhs)
    x_true = torch.randn(n, nrhs, dtype=torch.float64, device="cuda", generator=g)
    B = A @ x_true
    dA = devcopy(A)  # column-major A
    dB = devcopy(B)
    st, res = dp.gesv_ir_device(n, nrhs, dA, n, dB, n, precision=precision, max_iter=10,
                                tol=1e-14)
    assert st == 0
    assert res.info == n
    assert res.converged == 1
    assert res.backward_error <= 1e-14
    assert torch.equal(dA.T, A)  # A is not modified
    X = dB.T
    berr = (torch.linalg.norm(B - A @ X, float("inf"), dim=0) /
            (torch.linalg.norm(A, float("inf")) * torch.linalg.norm(X, float("inf"), dim=0) +
             torch.linalg.norm(B, float("inf"), dim=0))).max().item()
    assert berr <= 1e-14
    ferr = (torch.linalg.norm(X - x_true, float("inf")) / torch.linalg.norm(x_true, float("inf"))).item()
    assert ferr <= kappa * 1e-14
    if kappa >= 1e10:
        assert res.refactored == 1  # the mixed factors cannot carry kappa = 1e10
    if kappa <= 1e2 or (precision == dp.PRECISION_MIXED_BF16X6 and kappa <= 1e6):
        assert res.refactored == 0  # BF16x6 (about 2^-24) carries kappa up to 1e6


def test_fp64_ir_needs_at_most_few_steps():
    import delayed_pivoting as dp

    torch = _torch()
    n = 512
    A, g = conditioned(torch, n, 1e4, seed=5)
    B = A @ torch.randn(n, 3, dtype=torch.float64, device="cuda", generator=g)
    dA = devcopy(A)
    dB = devcopy(B)
    st, res = dp.gesv_ir_device(n, 3, dA, n, dB, n, precision=dp.PRECISION_FP64, max_iter=10,
                                tol=1e-14)
    assert st == 0 and res.converged == 1 and res.refactored == 0
    assert res.iterations <= 3


def test_mixed_factorisation_is_close():
    """The mixed-precision factors alone reconstruct A to about 1e-5 relative."""
    import delayed_pivoting as dp

    torch = _torch()
    n = 1024
    A, _ = conditioned(torch, n, 1e3, seed=3)
    d = devcopy(A)
    ipiv = np.zeros(n, dtype=np.int32)
    jpiv = np.zeros(n, dtype=np.int32)
    st, info = dp.getrf_device_ex(n, n, d, n, ipiv, jpiv, nb=64, nb_outer=256,
                                  precision=dp.PRECISION_MIXED_BF16X3)
    assert st == 0 and info == n
    F = d.T
    L = torch.tril(F, -1) + torch.eye(n, dtype=F.dtype, device=F.device)
    U = torch.triu(F)
    row = np.arange(n)
    col = np.arange(n)
    for k in range(n):
        row[[k, ipiv[k]]] = row[[ipiv[k], k]]
        col[[k, jpiv[k]]] = col[[jpiv[k], k]]
    PAQ = A[torch.from_numpy(row).cuda()][:, torch.from_numpy(col).cuda()]
    rel = (torch.linalg.norm(PAQ - L @ U) / torch.linalg.norm(A)).item()
    assert rel < 1e-4


def _conditioned(n, kappa, seed):
    """A = U diag(sigma) V^T, U and V orthogonal (QR of seeded N(0,1)), sigma
    geometric from 1 to 1/kappa; returns (A (host, Fortran), kappa_1(A))."""
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.logspace(0, -np.log10(kappa), n)
    a = np.asfortranarray((u * s) @ v.T)
    ainv = (v / s) @ u.T  # exact inverse of the construction
    k1 = np.abs(a).sum(axis=0).max() * np.abs(ainv).sum(axis=0).max()
    return a, k1


@pytest.mark.parametrize("n", [1, 70, 300])
@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_condest_brackets_kappa1(n, kappa):
    """Hager-Higham through FP64 factors: a lower bound of kappa_1 (up to
    rounding) and within a factor 10 of it (the estimator is exact for n = 1
    and usually within 3)."""
    import delayed_pivoting as dp

    torch = _torch()
    a, k1 = _conditioned(n, kappa, 100 + n)
    d_a = colmajor(torch, a)
    f = dp.Factor(n, d_a, n, precision=dp.PRECISION_FP64)
    st, est = f.condest()
    f.close()
    assert st == 0
    assert est <= k1 * (1 + 1e-4), (est, k1)  # solves through FP64 factors: kappa u <= 1e-6
    assert est >= k1 / 10.0, (est, k1)


def test_condest_of_singular_factorisation_is_infinite():
    import delayed_pivoting as dp

    torch = _torch()
    a = np.asfortranarray(np.random.default_rng(3).standard_normal((50, 50)))
    a[:, 7] = 0.0
    f = dp.Factor(50, colmajor(torch, a), 50, precision=dp.PRECISION_FP64)
    assert f.info()[0] < 50
    st, est = f.condest()
    f.close()
    assert st == 0 and est == float("inf")
