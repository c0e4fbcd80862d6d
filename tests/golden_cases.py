"""Loads the golden record fixtures (tests/golden/*.npz, written by
tests/golden/make_golden.py from the reference's own CPU code) and rebuilds
their inputs."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def names(max_elems: int | None = None):
    out = []
    for p in sorted(GOLDEN.glob("*.npz")):
        with np.load(p) as z:
            if max_elems is not None and int(z["m"]) * int(z["n"]) > max_elems:
                continue
        out.append(p.stem)
    return out


def load(name: str):
    """Returns (input matrix (Fortran, lda x n), case dict)."""
    import delayed_pivoting as dp

    with np.load(GOLDEN / f"{name}.npz") as z:
        case = {k: z[k] for k in z.files}
    for k in ("m", "n", "lda", "info", "policy"):
        case[k] = int(case[k])
    if str(case["kind"]) == "literal":
        a = np.asfortranarray(case["matrix"].astype(np.float64))
    else:
        a = dp.planted_matrix(case["m"], case["n"], int(case["seed"]), int(case["n_tiny"]),
                              int(case["n_zero"]), lda=case["lda"])
    return a, case
