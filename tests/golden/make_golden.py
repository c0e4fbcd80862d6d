"""Generates the golden record fixtures of the delayed-pivoting LU by running
the reference's own CPU code (delayed_lu/delayed_dgetrf.cpp and
delayed_dgetrf_column.cpp, compiled unmodified into oracle/_ref/ against
OpenBLAS).  Run from the repository root:

    python tests/golden/make_golden.py            # all cases except n=16384
    python tests/golden/make_golden.py --large    # also the n=16384 and n=32768 cases
    python tests/golden/make_golden.py --only config2_n32768   # one generated case

It also writes tests/golden/batch/config4_subset64.npz: the reference's
records for a seeded 64-matrix subset of the batched workload (orders
log-uniform in [32, 512], 0-2 exact-zero columns each).

Each case is written to tests/golden/<name>.npz with the inputs' recipe
(generator seed and planted columns, or the literal matrix for the reference's
own small known-answer cases), the reference's ipiv / jpiv / info, and its
scaled residual ||PAQ - LU||_F / (||A||_F * max(m,n) * u).
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "delayed-pivoting_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import delayed_pivoting as dp  # noqa: E402
import oracle as orc  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, m, n, lda, seed, n_tiny, n_zero, policy)
GENERATED = [
    ("config1_n1024", 1024, 1024, 1024, 12345, 16, 4, 0),
    ("config1_n1024_column", 1024, 1024, 1024, 12345, 16, 4, 1),
    ("tall_300x200", 300, 200, 310, 7, 2, 3, 0),
    ("wide_150x260", 150, 260, 150, 8, 1, 2, 0),
    ("square_70_zero2", 70, 70, 70, 9, 0, 2, 0),
    ("square_517_lda520", 517, 517, 520, 11, 3, 5, 0),
    ("square_2000_zero20", 2000, 2000, 2000, 21, 8, 20, 0),
    ("square_2000_zero20_column", 2000, 2000, 2000, 21, 8, 20, 1),
    ("single_1x1", 1, 1, 1, 3, 0, 0, 0),
    ("column_5x1", 5, 1, 5, 4, 0, 0, 0),
    ("row_1x6", 1, 6, 1, 5, 0, 0, 0),
    ("all_zero_9x9", 9, 9, 9, 6, 0, 9, 0),
]
LARGE = [("config2_n16384", 16384, 16384, 16384, 16384, 16, 3, 0),
         ("config2_n32768", 32768, 32768, 32768, 32768, 32, 6, 0)]
BATCH_SUBSET = ("config4_subset64", 64, 8192)  # (name, count, seed)


def reference_known_answer():
    """The reference's own known-answer inputs (delayed_lu_cuda/example.cu:115-143
    and delayed_lu/example.cpp:204-220), rebuilt from their description."""
    cases = []
    dense = np.array([[8.0, 1.0, 2.0, 0.0],
                      [2.0, 9.0, 1.0, 1.0],
                      [1.0, 1.0, 7.0, 2.0],
                      [0.0, 1.0, 1.0, 6.0]], order="F")
    cases.append(("ref_dense_4x4", dense, 4))
    rank3 = np.zeros((6, 6), order="F")
    rank3[2, 2], rank3[4, 4], rank3[5, 5] = 7.0, -5.0, 3.0
    cases.append(("ref_rank3_6x6", rank3, 3))
    rect = np.array([[5.0, 1.0, 0.0],
                     [1.0, 6.0, 1.0],
                     [0.0, 1.0, 7.0],
                     [1.0, 0.0, 1.0],
                     [0.0, 1.0, 0.0]], order="F")
    cases.append(("ref_rect_5x3", rect, 3))
    far = np.zeros((70, 70), order="F")
    far[0, 0], far[69, 69] = 100.0, 5.0
    cases.append(("ref_far_pivot_70", far, 2))
    diag = np.zeros((4096, 4096), order="F")
    for k in range(800):
        diag[k + 2, k + 2] = float(800 - k)
    cases.append(("ref_diag800_4096", diag, 800))
    return cases


def run_reference(a, m, n, policy):
    f = a.copy(order="F")
    fn = orc.ref_getrf if policy == 0 else orc.ref_getrf_column
    ipiv, jpiv, info = fn(f, m, n)
    res = orc.scaled_residual(a, f, m, n, info, ipiv, jpiv) if m * n <= 4096 * 4096 else -1.0
    return ipiv, jpiv, info, res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--large", action="store_true")
    ap.add_argument("--only", default=None, help="write only this generated case")
    args = ap.parse_args()
    orc.build(ref=True)
    if args.only:
        for case in GENERATED + LARGE:
            if case[0] == args.only:
                write_generated(*case)
                return
        raise SystemExit(f"no generated case {args.only}")
    for name, a, expect in reference_known_answer():
        m, n = a.shape
        ipiv, jpiv, info, res = run_reference(a, m, n, 0)
        assert info == expect, (name, info, expect)
        np.savez_compressed(OUT / f"{name}.npz", kind="literal", matrix=a, m=m, n=n, lda=m,
                            policy=0, ipiv=ipiv, jpiv=jpiv, info=info, scaled_residual=res)
        print(f"{name}: info={info} scaled_residual={res:.3g}")
    for case in GENERATED + (LARGE if args.large else []):
        write_generated(*case)
    batch_subset()


def write_generated(name, m, n, lda, seed, nt, nz, policy):
    a = dp.planted_matrix(m, n, seed, nt, nz, lda=lda)
    ipiv, jpiv, info, res = run_reference(a, m, n, policy)
    del a
    np.savez_compressed(OUT / f"{name}.npz", kind="generated", m=m, n=n, lda=lda, seed=seed,
                        n_tiny=nt, n_zero=nz, policy=policy, ipiv=ipiv, jpiv=jpiv, info=info,
                        scaled_residual=res)
    swaps = int((jpiv != np.arange(len(jpiv))).sum())
    print(f"{name}: info={info} column_swaps={swaps} scaled_residual={res:.3g}")


def batch_subset():
    name, count, seed = BATCH_SUBSET
    ns, n_zero = dp.batch_orders(count, seed)
    ipivs, jpivs, infos, worst = [], [], [], 0.0
    for i in range(count):
        n = int(ns[i])
        a = dp.batch_matrix(ns, n_zero, seed, i)
        ipiv, jpiv, info, res = run_reference(a, n, n, 0)
        ipivs.append(ipiv)
        jpivs.append(jpiv)
        infos.append(info)
        worst = max(worst, res)
    (OUT / "batch").mkdir(exist_ok=True)
    np.savez_compressed(OUT / "batch" / f"{name}.npz", count=count, seed=seed, ns=ns,
                        n_zero=n_zero, ipiv=np.concatenate(ipivs), jpiv=np.concatenate(jpivs),
                        info=np.array(infos, dtype=np.int32))
    delayed = int((np.array(infos) < ns).sum())
    print(f"{name}: {count} matrices, n in [{ns.min()}, {ns.max()}], {int(n_zero.sum())} zero "
          f"columns, {delayed} delayed, worst scaled_residual={worst:.3g}")


if __name__ == "__main__":
    main()
