"""Load generation for the request server (dp_server_*): a seeded stream of
factor+solve requests with follow-up solves, the device-resident matrices it
draws from, and an open-loop replay that submits requests at their arrival
times and collects the results with the server's own timestamps.

Matrices are A = U diag(sigma) V^T with U, V the Q factors of seeded N(0,1)
matrices and sigma geometric from 1 to 1/kappa, on a grid of orders and
condition numbers (a request draws its order log-uniformly and takes the
nearest grid order); right-hand sides are B = A X with X ~ N(0,1)."""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np


def grid_orders(lo=64, hi=8192, count=24):
    return sorted({int(round(v)) for v in np.exp(np.linspace(np.log(lo), np.log(hi), count))})


KAPPA_GRID = [float(v) for v in np.logspace(2, 6, 8)] + [1e10]


class MatrixPool:
    """Column-major device matrices for every (grid order, kappa) pair used by
    a stream.  pool[(n, kappa)] is an (n, n) tensor whose transpose is A."""

    def __init__(self, torch, pairs, seed=2025, device="cuda"):
        self.torch = torch
        self.mats = {}
        self.bytes = 0
        by_n = {}
        for n, kappa in sorted(set(pairs)):
            by_n.setdefault(n, []).append(kappa)
        for n, kappas in by_n.items():
            g = torch.Generator(device=device).manual_seed(seed * 100003 + n)
            u, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=device,
                                               generator=g))
            v, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=device,
                                               generator=g))
            for kappa in kappas:
                s = torch.logspace(0, -np.log10(kappa), n, dtype=torch.float64, device=device)
                a = (u * s) @ v.T
                self.mats[(n, kappa)] = a.T.contiguous()  # column-major storage of A
                self.bytes += 8 * n * n
            del u, v
        torch.cuda.synchronize()

    def __getitem__(self, key):
        return self.mats[key]


@dataclass
class Solve:
    rid: int
    nrhs: int
    factor_id: int = 0  # 0: the request's own factorisation


@dataclass
class Req:
    rid: int
    n: int
    kappa: float
    solves: list = field(default_factory=list)  # first: factor+solve, then follow-ups


def make_stream(count, seed, lo=64, hi=8192, p_ill=0.1, kappa_lo=1e2, kappa_hi=1e6,
                max_rhs=32, max_followups=4):
    """The served workload: orders log-uniform in [lo, hi] snapped to the grid,
    kappa log-uniform in [kappa_lo, kappa_hi] snapped to KAPPA_GRID (1 - p_ill)
    or 1e10 (p_ill), 1..max_rhs right-hand sides, 0..max_followups follow-up
    solves of 1..max_rhs right-hand sides each."""
    rng = np.random.default_rng(seed)
    orders = np.array(grid_orders(lo, hi))
    kgrid = np.array(KAPPA_GRID[:-1])
    reqs = []
    rid = 1
    for _ in range(count):
        n = int(orders[np.argmin(np.abs(np.log(orders) - rng.uniform(np.log(lo), np.log(hi))))])
        if rng.uniform() < p_ill:
            kappa = 1e10
        else:
            lk = rng.uniform(np.log(kappa_lo), np.log(kappa_hi))
            kappa = float(kgrid[np.argmin(np.abs(np.log(kgrid) - lk))])
        q = Req(rid, n, kappa)
        q.solves.append(Solve(rid, int(rng.integers(1, max_rhs + 1))))
        for j in range(int(rng.integers(0, max_followups + 1))):
            q.solves.append(Solve(rid + 1 + j, int(rng.integers(1, max_rhs + 1)), factor_id=rid))
        rid += len(q.solves) + 1
        reqs.append(q)
    return reqs


class RhsSet:
    """Pristine right-hand sides of every solve of a stream (device), and the
    work buffers the server overwrites with the solutions."""

    def __init__(self, torch, pool, reqs, seed=7):
        g = torch.Generator(device="cuda").manual_seed(seed)
        self.src, self.work = {}, {}
        self.bytes = 0
        for q in reqs:
            A = pool[(q.n, q.kappa)].T
            for s in q.solves:
                X = torch.randn(q.n, s.nrhs, dtype=torch.float64, device="cuda", generator=g)
                b = (A @ X).T.contiguous()  # column-major n x nrhs
                self.src[s.rid] = b
                self.work[s.rid] = torch.empty_like(b)
                self.bytes += 8 * q.n * s.nrhs
        torch.cuda.synchronize()

    def reset(self, torch):
        for k, b in self.src.items():
            self.work[k].copy_(b)
        torch.cuda.synchronize()


def replay(server, pool, rhs, reqs, rate=None, seed=11, timeout=600.0):
    """Submits every request (and its follow-ups, at the same arrival time) at
    Poisson arrival times of `rate` requests/s (None: all at once) and waits
    for every result.  Returns (results by id, first submit, last completion)
    in the server's clock."""
    from .api import server_clock

    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(reqs)) if rate else np.zeros(len(reqs))
    arrivals = np.cumsum(gaps) - (gaps[0] if len(gaps) else 0.0)
    total = sum(len(q.solves) for q in reqs)
    results = {}
    done = threading.Event()
    errors = []

    def poller():
        while len(results) < total:
            for r in server.poll(1024, wait_ms=20):
                results[r.id] = r
            if time.monotonic() - t_start > timeout:
                errors.append("timeout")
                break
        done.set()

    t_start = time.monotonic()
    th = threading.Thread(target=poller, daemon=True)
    th.start()
    t0 = server_clock()
    for q, at in zip(reqs, arrivals):
        while True:
            now = server_clock() - t0
            if now >= at:
                break
            if at - now > 0.002:
                time.sleep(at - now - 0.001)
        A = pool[(q.n, q.kappa)]
        for s in q.solves:
            b = rhs.work[s.rid]
            if s.factor_id == 0:
                st = server.submit(s.rid, q.n, A, q.n, b, q.n, s.nrhs,
                                   followups=len(q.solves) - 1)
            else:
                st = server.submit(s.rid, q.n, None, q.n, b, q.n, s.nrhs, factor_id=s.factor_id)
            if st != 0:
                errors.append(f"submit {s.rid}: status {st}")
    done.wait()
    th.join()
    if errors:
        raise RuntimeError("; ".join(errors[:5]))
    first = min(r.t_submit for r in results.values())
    last = max(r.t_done for r in results.values())
    return results, first, last
