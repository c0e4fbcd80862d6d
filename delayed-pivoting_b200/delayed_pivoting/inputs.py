"""Seeded synthetic inputs (lib/libdp_matgen.so): N(0,1) column-major
matrices from MT19937-64 with planted tiny and exact-zero columns."""
from __future__ import annotations

import numpy as np

from .api import matgen


def mt64_nth(seed: int, count: int) -> int:
    return int(matgen().dpgen_mt64_nth(seed, count))


def normal_matrix(m: int, n: int, seed: int, lda: int | None = None) -> np.ndarray:
    """(lda x n) Fortran-ordered float64 array; rows [0, m) ~ N(0,1), padding rows 0."""
    lda = m if lda is None else lda
    a = np.zeros((max(lda, 1), n), dtype=np.float64, order="F")
    if m > 0 and n > 0:
        matgen().dpgen_normal_matrix(m, n, a.ctypes.data, lda, seed)
    return a


def plant_columns(a: np.ndarray, m: int, n: int, seed: int, n_tiny: int, n_zero: int,
                  tiny_scale: float = 1e-18):
    lda = a.shape[0]
    tiny = np.zeros(max(n_tiny, 1), dtype=np.int32)
    zero = np.zeros(max(n_zero, 1), dtype=np.int32)
    rc = matgen().dpgen_plant_columns(m, n, a.ctypes.data, lda, seed, n_tiny, tiny_scale, n_zero,
                                      tiny.ctypes.data, zero.ctypes.data)
    if rc != 0:
        raise ValueError("bad planted-column counts")
    return tiny[:n_tiny], zero[:n_zero]


def planted_matrix(m: int, n: int, seed: int, n_tiny: int = 0, n_zero: int = 0,
                   tiny_scale: float = 1e-18, lda: int | None = None) -> np.ndarray:
    """N(0,1) matrix with planted tiny and exact-zero columns (the reference's
    workload: configs of n = 1024 with 16 tiny + 4 zero, n = 16384 with 0.1 %
    tiny and 0.02 % zero)."""
    a = normal_matrix(m, n, seed, lda)
    plant_columns(a, m, n, seed, n_tiny, n_zero, tiny_scale)
    return a


def uniform_stream(count: int, seed: int) -> np.ndarray:
    out = np.empty(count, dtype=np.float64)
    if count:
        matgen().dpgen_uniform(out.ctypes.data, count, seed)
    return out


def normal_vector(count: int, seed: int) -> np.ndarray:
    out = np.empty(count, dtype=np.float64)
    if count:
        matgen().dpgen_normal_vector(out.ctypes.data, count, seed)
    return out


# ---- batches of small matrices -------------------------------------------

def batch_orders(count: int, seed: int, lo: int = 32, hi: int = 512, p_zero: float = 0.3):
    """Orders log-uniform in [lo, hi] and, per matrix, 0-2 exact-zero columns
    (two independent draws with probability p_zero each).  Returns (ns, n_zero)
    as int32 arrays."""
    u = uniform_stream(3 * count, seed).reshape(count, 3) if count else np.zeros((0, 3))
    ns = np.floor(np.exp(np.log(lo) + u[:, 0] * (np.log(hi + 1) - np.log(lo))))
    ns = np.clip(ns, lo, hi).astype(np.int32)
    n_zero = (u[:, 1] < p_zero).astype(np.int32) + (u[:, 2] < p_zero).astype(np.int32)
    return ns, n_zero.astype(np.int32)


def batch_matrix_seed(seed: int, i: int) -> int:
    return (seed * 1_000_003 + i) & 0xFFFFFFFFFFFFFFFF


def fill_batch(buf: np.ndarray, offsets, ns, n_zero, seed: int) -> None:
    """Writes matrix i (N(0,1), n_zero[i] planted exact-zero columns, column-major,
    lda = ns[i]) at element offsets[i] of the float64 host buffer `buf`."""
    G = matgen()
    assert buf.dtype == np.float64 and buf.flags.c_contiguous
    base = buf.ctypes.data
    scratch = np.zeros(4, dtype=np.int32)
    for i, (n, off, nz) in enumerate(zip(ns, offsets, n_zero)):
        n, off, nz = int(n), int(off), int(nz)
        assert off + n * n <= buf.size
        ptr = base + 8 * off
        s = batch_matrix_seed(seed, i)
        G.dpgen_normal_matrix(n, n, ptr, n, s)
        if nz:
            rc = G.dpgen_plant_columns(n, n, ptr, n, s, 0, 1e-18, nz, scratch.ctypes.data,
                                       scratch[2:].ctypes.data)
            if rc != 0:
                raise ValueError("bad planted-column counts")


def batch_matrix(ns, n_zero, seed: int, i: int) -> np.ndarray:
    """Matrix i of fill_batch as an (n x n) Fortran array."""
    n = int(ns[i])
    return planted_matrix(n, n, batch_matrix_seed(seed, i), 0, int(n_zero[i]))


def symmetric_matrix(n: int, seed: int, lda: int | None = None, zero_nodes=(),
                     zero_diag: bool = False) -> np.ndarray:
    """Seeded symmetric indefinite matrix for the LDL^T path (Fortran, lda >=
    n): N(0, 1) entries of NumPy's PCG64 stream (default_rng(seed)), the lower
    triangle mirrored to the upper; `zero_nodes` rows / columns cleared (they
    can only be delayed), `zero_diag` clears the diagonal."""
    lda = n if lda is None else lda
    x = np.random.default_rng(seed).standard_normal((n, n))
    a = np.tril(x) + np.tril(x, -1).T
    if zero_diag:
        np.fill_diagonal(a, 0.0)
    for z in zero_nodes:
        a[z, :] = 0.0
        a[:, z] = 0.0
    out = np.zeros((lda, n), order="F")
    out[:n, :n] = a
    return out
