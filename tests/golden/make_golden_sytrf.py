"""Generates the golden record fixtures of the delayed Bunch-Kaufman LDL^T by
running the reference's own CPU code (delayed-bunch-kaufman/
delayed_sytrf_blocked.cpp and delayed_sytrf.cpp, compiled unmodified into
oracle/_ref/libref_delayed_bk.so against OpenBLAS).  Run from the repository
root:

    python tests/golden/make_golden_sytrf.py            # the 15 fixtures below
    python tests/golden/make_golden_sytrf.py --large    # also large/sym_16384.npz

Each case is written to tests/golden/sytrf/<name>.npz with the input's recipe
(size, leading dimension, generator seed, zeroed nodes, cleared diagonal, or
the reference's own rank-8 known-answer matrix), the blocked reference's
perm / piv_size / info, and the largest |P A P^T - L D L^T|.  The unblocked
reference must give the same records, or the case is rejected (it would be
order-sensitive between two builds of the reference itself).

--large writes tests/golden/sytrf/large/sym_16384.npz from the blocked
reference alone (the unblocked one, BLAS-2 throughout, is impractically slow
at that order); with --check-oracle the restatement is run on it as well
(a few minutes on 8 cores) and must give the same records.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))

import oracle as orc  # noqa: E402

OUT = Path(__file__).resolve().parent / "sytrf"

# (name, n, lda, seed, zero_nodes, zero_diag)
CASES = [
    ("single_1", 1, 1, 1, (), False),
    ("single_zero_1", 1, 1, 1, (0,), False),
    ("pair_2_zero_diag", 2, 2, 2, (), True),
    ("all_zero_9", 9, 9, 3, tuple(range(9)), False),
    ("sym_7", 7, 7, 1, (), False),
    ("sym_65", 65, 65, 4, (), False),
    ("sym_200", 200, 200, 2, (), False),
    ("sym_300_zero2", 300, 300, 3, (5, 77), False),
    ("zero_diag_150", 150, 150, 4, (), True),
    ("zero_diag_257_zero3", 257, 257, 6, (0, 1, 2), True),
    ("sym_333_lda340", 333, 340, 7, (40,), False),
    ("sym_1000", 1000, 1000, 5, (), False),
    ("sym_2048_zero8", 2048, 2048, 8, (3, 100, 511, 512, 1000, 1500, 2000, 2047), False),
    ("sym_4096", 4096, 4096, 4096, (), False),
]


def large(check_oracle: bool) -> None:
    out = OUT / "large"
    out.mkdir(parents=True, exist_ok=True)
    n = 16384
    a = orc.sym_matrix(n, n)
    f = a.copy(order="F")
    perm, piv, info = orc.ref_sytrf(f, "blocked")
    del f
    if check_oracle:
        g = a.copy(order="F")
        p2, v2, i2 = orc.oracle_sytrf(g)
        if not (np.array_equal(perm, p2) and np.array_equal(piv, v2) and info == i2):
            raise SystemExit("sym_16384: the restatement's records differ from the reference's")
    np.savez_compressed(out / f"sym_{n}.npz", perm=perm, piv_size=piv, info=np.int32(info),
                        n=n, lda=n, seed=n, zero_nodes=np.zeros(0, np.int32), zero_diag=False,
                        rank8=False, max_error=np.float64(np.nan))
    print(f"large/sym_{n}: info={info} 2x2={int((piv == 2).sum())}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--large", action="store_true")
    ap.add_argument("--check-oracle", action="store_true")
    args = ap.parse_args()
    if args.large:
        large(args.check_oracle)
        return
    OUT.mkdir(exist_ok=True)
    cases = [(name, dict(n=n, lda=lda, seed=seed, zero_nodes=np.array(z, dtype=np.int32),
                         zero_diag=zd, rank8=False))
             for name, n, lda, seed, z, zd in CASES]
    cases.append(("rank8_4096", dict(n=4096, lda=4096, seed=0, zero_nodes=np.zeros(0, np.int32),
                                     zero_diag=False, rank8=True)))
    for name, r in cases:
        a = (orc.rank8_example(r["n"]) if r["rank8"] else
             orc.sym_matrix(r["n"], r["seed"], r["lda"], tuple(r["zero_nodes"]), r["zero_diag"]))
        f = a.copy(order="F")
        perm, piv, info = orc.ref_sytrf(f, "blocked")
        g = a.copy(order="F")
        perm_u, piv_u, info_u = orc.ref_sytrf(g, "unblocked")
        if not (np.array_equal(perm, perm_u) and np.array_equal(piv, piv_u) and info == info_u):
            raise SystemExit(f"{name}: blocked and unblocked reference records differ")
        res = orc.ldl_residual(a, f, perm, piv, info)
        np.savez_compressed(OUT / f"{name}.npz", perm=perm, piv_size=piv, info=np.int32(info),
                            max_error=np.float64(res), **r)
        print(f"{name}: n={r['n']} info={info} 2x2={int((piv == 2).sum())} max_err={res:.2e}")


if __name__ == "__main__":
    main()
