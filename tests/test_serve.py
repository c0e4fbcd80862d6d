"""Tests of the serving layer: resident factorisations (dp_factor_*) and the
request server (dp_server_*).

Matrices are A = U diag(sigma) V^T with U, V from the QR of seeded N(0,1)
matrices and sigma geometric from 1 to 1/kappa; right-hand sides B = A X_true.
Every solve must reach a normwise backward error <= 1e-14 (the server's
tolerance); kappa = 1e10 must end on FP64 factors (the mixed-precision
refinement stalls and the request is re-factored in FP64); each request's
result must be the same alone and among others, within the stated tolerance
(backward error <= 1e-14; bitwise on the batched small-request path)."""
import time

import numpy as np
import pytest

import delayed_pivoting as dp

TOL = 1e-14


def test_server_options_defaults():
    o = dp.server_options()
    assert o.budget_bytes == 160 << 30
    assert o.precision == dp.PRECISION_MIXED_BF16X6
    assert o.small_max_n == dp.BATCH_MAX_N and o.max_iter == 10 and o.tol == TOL
    assert o.mixed_min_n == 12288  # mixed factors only where they beat FP64


def test_server_rejects_bad_mixed_min_n_before_device_work():
    import ctypes

    h = ctypes.c_void_p()
    o = dp.server_options(mixed_min_n=-2)
    assert dp.lib().dp_server_create(ctypes.byref(h), ctypes.byref(o)) == dp.INVALID_ARGUMENT


# ---------------------------------------------------------------- GPU ----

def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def conditioned(torch, n, kappa, seed):
    """Column-major device copy of U diag(sigma) V^T (as a (n, n) tensor whose
    transpose is the matrix) and a generator for the right-hand sides."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    u, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    v, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    sigma = torch.logspace(0, -np.log10(kappa), n, dtype=torch.float64, device="cuda")
    A = (u * sigma) @ v.T
    return A, g


def colmajor(t):
    return t.T.contiguous().clone()


def backward_error(torch, A, X, B):
    r = B - A @ X
    den = (torch.linalg.norm(A, float("inf")) * torch.linalg.norm(X, float("inf"), dim=0) +
           torch.linalg.norm(B, float("inf"), dim=0))
    return (torch.linalg.norm(r, float("inf"), dim=0) / den).max().item()


@pytest.mark.gpu
def test_resident_factor_serves_several_solves():
    torch = _torch()
    n = 700
    A, g = conditioned(torch, n, 1e4, 11)
    dA = colmajor(A)
    f = dp.Factor(n, dA, n, precision=dp.PRECISION_MIXED_BF16X3)
    info, prec, _ = f.info()
    assert info == n and prec == dp.PRECISION_MIXED_BF16X3
    for nrhs in (1, 5, 33):
        Xt = torch.randn(n, nrhs, dtype=torch.float64, device="cuda", generator=g)
        B = A @ Xt
        dB = colmajor(B)
        st, res = f.solve(dB, n, nrhs)
        assert st == 0 and res.converged == 1 and res.backward_error <= TOL
        X = dB.T
        assert backward_error(torch, A, X, B) <= TOL
        assert torch.equal(dA.T, A)  # the matrix is untouched
    assert f.info()[1] == dp.PRECISION_MIXED_BF16X3
    f.close()


@pytest.mark.gpu
def test_resident_factor_ill_conditioned_goes_fp64():
    torch = _torch()
    n = 600
    A, g = conditioned(torch, n, 1e10, 12)
    dA = colmajor(A)
    f = dp.Factor(n, dA, n, precision=dp.PRECISION_MIXED_BF16X3)
    B = A @ torch.randn(n, 3, dtype=torch.float64, device="cuda", generator=g)
    dB = colmajor(B)
    st, res = f.solve(dB, n, 3)
    assert st == 0 and res.refactored == 1 and res.backward_error <= TOL
    assert f.info()[1] == dp.PRECISION_FP64
    # the next solve runs on the FP64 factors directly
    dB2 = colmajor(B)
    st, res2 = f.solve(dB2, n, 3)
    assert st == 0 and res2.refactored == 1 and res2.factor_ms == 0.0 and res2.backward_error <= TOL
    f.close()


def make_requests(torch, seed, sizes, kappas):
    """Requests (dicts) with device matrices and right-hand sides; follow-ups
    get their own right-hand sides."""
    rng = np.random.default_rng(seed)
    reqs = []
    rid = 1
    for i, n in enumerate(sizes):
        kappa = kappas[i % len(kappas)]
        A, g = conditioned(torch, n, kappa, seed * 1000 + i)
        nf = int(rng.integers(0, 3))
        rhs = []
        for _ in range(1 + nf):
            k = int(rng.integers(1, 9))
            rhs.append(A @ torch.randn(n, k, dtype=torch.float64, device="cuda", generator=g))
        reqs.append(dict(id=rid, n=n, kappa=kappa, A=A, dA=colmajor(A), rhs=rhs,
                         ids=[rid] + [rid + 1 + j for j in range(nf)]))
        rid += 2 + nf
    return reqs


def run_server(server, reqs, together=True, timeout=300.0):
    """Submits every request and its follow-ups; returns {id: (result, X)}."""
    outs = {}
    bufs = {}

    def wait_for(ids):
        t0 = time.time()
        while not ids.issubset(outs) and time.time() - t0 < timeout:
            for r in server.poll(256, wait_ms=50):
                outs[r.id] = r
        assert ids.issubset(outs), "server did not finish"

    import torch

    for q in reqs:
        for rid, B in zip(q["ids"], q["rhs"]):
            bufs[rid] = colmajor(B)
    # the server's streams do not wait for the caller's: inputs must be
    # complete on the device when they are submitted
    torch.cuda.synchronize()
    pending_follow = []
    for q in reqs:
        n = q["n"]
        for j, (rid, B) in enumerate(zip(q["ids"], q["rhs"])):
            dB = bufs[rid]
            if j == 0:
                st = server.submit(rid, n, q["dA"], n, dB, n, B.shape[1],
                                   followups=len(q["ids"]) - 1)
                assert st == 0
                if not together:
                    wait_for({rid})
            else:
                pending_follow.append((rid, q, dB, B.shape[1]))
                if not together:
                    assert server.submit(rid, n, None, n, dB, n, B.shape[1],
                                         factor_id=q["id"]) == 0
                    wait_for({rid})
    if together:
        for rid, q, dB, k in pending_follow:
            assert server.submit(rid, q["n"], None, q["n"], dB, q["n"], k, factor_id=q["id"]) == 0
        wait_for({rid for q in reqs for rid in q["ids"]})
    return {rid: (outs[rid], bufs[rid].T.clone()) for rid in outs}


SIZES = [16, 40, 64, 100, 200, 300, 511, 513, 700, 1200, 37, 450, 900]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [dp.PRECISION_MIXED_BF16X6, dp.PRECISION_MIXED_BF16X3,
                                       dp.PRECISION_FP64])
def test_server_mixed_stream(precision):
    torch = _torch()
    reqs = make_requests(torch, 3, SIZES, [1e2, 1e5, 1e10])
    # mixed factors for every blocked order (the default keeps FP64 below 12288)
    srv = dp.Server(precision=precision, large_workers=3, mixed_min_n=-1)
    out = run_server(srv, reqs)
    st = srv.stats()
    srv.close()
    for q in reqs:
        for rid, B in zip(q["ids"], q["rhs"]):
            r, X = out[rid]
            assert r.status == 0 and r.info == q["n"], (q["n"], rid)
            assert r.backward_error <= TOL, (q["n"], q["kappa"], r.backward_error)
            assert backward_error(torch, q["A"], X, B) <= 2 * TOL
            assert r.path == (0 if q["n"] <= 512 else 1)
            assert r.t_submit <= r.t_admit <= r.t_start <= r.t_done
        r0 = out[q["id"]][0]
        if q["n"] > 512 and precision != dp.PRECISION_FP64:
            if q["kappa"] >= 1e10:
                assert r0.precision == dp.PRECISION_FP64 and r0.refactored == 1
            elif q["kappa"] <= 1e2 or (precision == dp.PRECISION_MIXED_BF16X6 and q["kappa"] <= 1e5):
                assert r0.precision == precision
    assert st.small_launches >= 1 and st.small_items > 0 and st.large_items > 0
    assert st.residents == 0 and st.bytes_in_use == 0


@pytest.mark.gpu
def test_server_routes_orders_below_mixed_min_n_to_fp64():
    """A mixed server factors blocked requests of order < mixed_min_n in FP64
    and the others in mixed precision; both meet the backward-error target."""
    torch = _torch()
    reqs = make_requests(torch, 9, [600, 900], [1e2])
    srv = dp.Server(precision=dp.PRECISION_MIXED_BF16X6, large_workers=2, mixed_min_n=800)
    out = run_server(srv, reqs)
    srv.close()
    for q in reqs:
        r0 = out[q["id"]][0]
        assert r0.status == 0 and r0.backward_error <= TOL
        want = dp.PRECISION_FP64 if q["n"] < 800 else dp.PRECISION_MIXED_BF16X6
        assert r0.precision == want, (q["n"], r0.precision)
    srv = dp.Server(precision=dp.PRECISION_MIXED_BF16X6, large_workers=2)  # default 12288
    out = run_server(srv, make_requests(torch, 10, [900], [1e2]))
    srv.close()
    assert all(r.precision == dp.PRECISION_FP64 for r, _ in out.values())


@pytest.mark.gpu
def test_server_result_alone_equals_result_in_mix():
    """Each request alone (submitted and awaited one by one: no follow-up is
    coalesced) and in the mix (all at once: a factorisation's follow-ups are
    solved together in one refined multi-RHS solve) meets the stated
    tolerance - normwise backward error <= 1e-14, recomputed here from the
    returned X - and the two solutions agree to what that tolerance allows
    (forward difference <= 2 kappa 1e-14).  Small requests (batched path, no
    coalescing) stay bitwise equal."""
    torch = _torch()
    reqs = make_requests(torch, 5, SIZES, [1e3, 1e6, 1e10])
    srv = dp.Server(precision=dp.PRECISION_MIXED_BF16X6, large_workers=4, mixed_min_n=-1)
    alone = run_server(srv, reqs, together=False)
    mix = run_server(srv, reqs, together=True)
    srv.close()
    assert set(alone) == set(mix)
    by_id = {rid: (q, j) for q in reqs for j, rid in enumerate(q["ids"])}
    for rid in alone:
        ra, Xa = alone[rid]
        rm, Xm = mix[rid]
        assert ra.status == rm.status == 0
        assert ra.backward_error <= TOL and rm.backward_error <= TOL, rid
        q, j = by_id[rid]
        A, B = q["A"], q["rhs"][j]
        for X in (Xa, Xm):  # independent check (cuBLAS residual: its own rounding)
            berr = (torch.linalg.norm(B - A @ X, float("inf"), dim=0) /
                    (torch.linalg.norm(A, float("inf")) * torch.linalg.norm(X, float("inf"), dim=0)
                     + torch.linalg.norm(B, float("inf"), dim=0))).max().item()
            assert berr <= 2 * TOL, (rid, berr)
        diff = (Xa - Xm).abs().max().item() / Xa.abs().max().item()
        assert diff <= 2 * q["kappa"] * TOL, (rid, diff)
        if q["n"] <= dp.BATCH_MAX_N:
            assert torch.equal(Xa, Xm), rid


@pytest.mark.gpu
def test_server_respects_the_budget():
    torch = _torch()
    budget = 40 << 20
    reqs = make_requests(torch, 7, [600, 650, 700, 750, 800, 300, 200, 520], [1e3])
    srv = dp.Server(precision=dp.PRECISION_FP64, large_workers=4, budget_bytes=budget)
    # a request that can never fit is refused at once
    big = torch.zeros(2500 * 2500, dtype=torch.float64, device="cuda")
    rhs = torch.zeros(2500, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert srv.submit(999999, 2500, big, 2500, rhs, 2500, 1) == dp.INVALID_ARGUMENT
    out = run_server(srv, reqs)
    st = srv.stats()
    srv.close()
    assert all(r.status == 0 and r.backward_error <= TOL for r, _ in out.values())
    assert 0 < st.bytes_peak <= budget


@pytest.mark.gpu
def test_server_follow_up_errors():
    torch = _torch()
    n = 100
    A, g = conditioned(torch, n, 1e2, 9)
    dA = colmajor(A)
    srv = dp.Server()
    b = colmajor(A @ torch.randn(n, 1, dtype=torch.float64, device="cuda", generator=g))
    torch.cuda.synchronize()
    # unknown factorisation
    assert srv.submit(5, n, None, n, b, n, 1, factor_id=77) == dp.INVALID_ARGUMENT
    # bad arguments
    assert srv.submit(0, n, dA, n, b, n, 1) == dp.INVALID_ARGUMENT
    assert srv.submit(6, n, dA, n - 1, b, n, 1) == dp.INVALID_ARGUMENT
    assert srv.submit(6, n, dA, n, b, n, 65) == dp.INVALID_ARGUMENT
    # one declared follow-up: the second is refused
    assert srv.submit(10, n, dA, n, b, n, 1, followups=1) == 0
    assert srv.submit(10, n, dA, n, b, n, 1) == dp.INVALID_ARGUMENT  # duplicate live id
    b1 = colmajor(A @ torch.randn(n, 1, dtype=torch.float64, device="cuda", generator=g))
    b2 = colmajor(A @ torch.randn(n, 1, dtype=torch.float64, device="cuda", generator=g))
    torch.cuda.synchronize()
    assert srv.submit(11, n, None, n, b1, n, 1, factor_id=10) == 0
    outs = {}
    t0 = time.time()
    while len(outs) < 2 and time.time() - t0 < 60:
        for r in srv.poll(16, wait_ms=50):
            outs[r.id] = r
    assert outs[10].status == 0 and outs[11].status == 0
    assert srv.submit(12, n, None, n, b2, n, 1, factor_id=10) == dp.INVALID_ARGUMENT
    assert srv.stats().residents == 0
    srv.close()


@pytest.mark.gpu
def test_server_singular_request_reports_info():
    torch = _torch()
    n = 300
    A = torch.randn(n, n, dtype=torch.float64, device="cuda")
    A[:, 7] = 0.0
    for size, path in ((n, 0), (900, 1)):
        M = torch.randn(size, size, dtype=torch.float64, device="cuda")
        M[:, 7] = 0.0
        dM = colmajor(M)
        b = torch.ones(size, 1, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        srv = dp.Server(precision=dp.PRECISION_FP64)
        assert srv.submit(1, size, dM, size, b, size, 1) == 0
        res = []
        t0 = time.time()
        while not res and time.time() - t0 < 60:
            res = srv.poll(1, wait_ms=50)
        srv.close()
        assert res[0].status == 0 and res[0].info == size - 1 and res[0].path == path
