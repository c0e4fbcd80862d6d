"""Python access to the two CPU checkers of the delayed-pivoting LU.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU leg of bench.py, never by the product library.

* ``oracle_getrf`` - the plain-C restatement (delayed_getrf_oracle.c) of
  delayed_lu/delayed_dgetrf.cpp:129-251 and delayed_dgetrf_column.cpp:99-211,
  with a panel width and an acceptance threshold.
* ``ref_getrf`` / ``ref_getrf_column`` / ``ref_lapack_getrf`` - the reference's
  own unmodified CPU sources compiled against SciPy's bundled OpenBLAS into
  ``_ref/libref_delayed_lu.so`` by the Makefile beside this file.
* ``residual`` - ||P A Q - Lbar Ubar||_F and ||A||_F of a compact factor, the
  reconstruction check of delayed_lu_cuda/example.cu:24-80.
* ``oracle_front`` - the multifrontal hand-off (partial factorisation of a
  front with p fully-summed rows / columns, contribution block), restated
  from the reference's design document (doc/...LU方法.md:228-457; the
  reference has no code for it): the fully-summed block by ``oracle_getrf``,
  the rest in NumPy.  Only its first step is pinned by the reference; the
  rest is checked against the Schur-complement identity in the tests.
* ``oracle_sytrf`` - the plain-C restatement (delayed_sytrf_oracle.c) of the
  blocked delayed Bunch-Kaufman LDL^T
  (delayed-bunch-kaufman/delayed_sytrf_blocked.cpp:141-358), panel width a
  parameter; ``ref_sytrf`` - the reference's own ``delayed_sytrf`` /
  ``delayed_sytrf_blocked`` / ``lapack_sytrf`` compiled into
  ``_ref/libref_delayed_bk.so``; ``ldl_residual`` - the reconstruction check
  of delayed-bunch-kaufman/example.cpp:97-160 (P A P^T against L D L^T with
  the delayed Schur complement as D's trailing block).
* ``_ref/ref_cuda_benchmark`` / ``_ref/ref_cuda_example`` - the reference's own
  GPU build (cuBLAS), and ``_ref/benchmark_on_b200`` / ``_ref/example_on_b200``
  - the same unmodified callers linked against libdelayed_lu_b200.so; see
  ``ref_binary``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle_dp.so"
REF_SO = HERE / "_ref" / "libref_delayed_lu.so"
REF_BK_SO = HERE / "_ref" / "libref_delayed_bk.so"

_or = None
_ref = None
_refbk = None


def build(ref: bool = True) -> None:
    """Compiles the oracle (and, when the reference tree exists, the reference)."""
    targets = ["oracle"]
    if ref and Path(os.environ.get("DP_REFERENCE", "/root/reference")).exists():
        targets += ["ref", "refgpu", "refbk"]
    env = dict(os.environ)
    if "DP_REFERENCE" in os.environ:
        env["REF"] = os.environ["DP_REFERENCE"]
    subprocess.run(["make", "-s", "-C", str(HERE)] + targets, check=True, env=env)


def _ip():
    return ctypes.POINTER(ctypes.c_int)


def oracle_lib() -> ctypes.CDLL:
    global _or
    if _or is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"oracle not built: {ORACLE_SO}")
        L = ctypes.CDLL(str(ORACLE_SO))
        L.oracle_delayed_getrf.restype = ctypes.c_int
        L.oracle_delayed_getrf.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.c_int, _ip(), _ip(), _ip(), ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int]
        L.oracle_residual.restype = None
        L.oracle_residual.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip(), _ip(),
                                      ctypes.c_void_p, _ip(), _ip(), ctypes.c_void_p]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_sytrf.restype = ctypes.c_int
        L.oracle_sytrf.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _ip(), _ip(),
                                   ctypes.c_int]
        _or = L
    return _or


def ref_available() -> bool:
    return REF_SO.exists()


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise RuntimeError(f"reference CPU build missing: {REF_SO}")
        L = ctypes.CDLL(str(REF_SO))
        for name in ("ref_delayed_getrf", "ref_delayed_getrf_column"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _ip(), _ip(),
                          _ip()]
        L.ref_lapack_getrf.restype = None
        L.ref_lapack_getrf.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                       _ip(), _ip()]
        L.ref_set_threads.restype = None
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_get_threads.restype = ctypes.c_int
        _ref = L
    return _ref


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _check(a):
    assert a.dtype == np.float64 and a.flags.f_contiguous


def oracle_getrf(a: np.ndarray, m: int | None = None, n: int | None = None, nb: int = 64,
                 threshold: float = 0.0, policy: int = 0):
    """Factors `a` (Fortran float64, lda = a.shape[0]) in place.
    Returns (ipiv, jpiv, info)."""
    _check(a)
    lda = a.shape[0]
    m = lda if m is None else m
    n = a.shape[1] if n is None else n
    piv = max(min(m, n), 1)
    ipiv = np.zeros(piv, dtype=np.int32)
    jpiv = np.zeros(piv, dtype=np.int32)
    info = ctypes.c_int(-1)
    oracle_lib().oracle_delayed_getrf(m, n, a.ctypes.data, lda, _p(ipiv), _p(jpiv),
                                      ctypes.byref(info), nb, threshold, policy)
    k = min(m, n)
    return ipiv[:k], jpiv[:k], info.value


def _composite(rec, size):
    src = np.arange(size)
    for k, r in enumerate(rec):
        src[[k, r]] = src[[r, k]]
    return src


def oracle_front(f: np.ndarray, p: int):
    """Partial delayed LU of the front `f` (m x n, Fortran float64) whose
    leading p rows / columns are fully summed; returns (npiv, ipiv, jpiv,
    out) with `out` the factored front: its first npiv rows / columns L and
    U, out[npiv:, npiv:] the contribution block (the delayed rows / columns of
    the fully-summed block first).  Pivots only inside the fully-summed block
    (delayed_getrf on f[:p, :p]), then its permutations, U12 = L11^-1 F12,
    L21 = F21 U11^-1 and the Schur updates of the delayed rows / columns and
    of F22, in the order the device applies them."""
    m, n = f.shape
    out = np.array(f, dtype=np.float64, order="F", copy=True)
    if p == 0:
        return 0, np.zeros(0, np.int32), np.zeros(0, np.int32), out
    f11 = np.asfortranarray(out[:p, :p])
    ipiv, jpiv, k = oracle_getrf(f11, p, p, nb=64)
    out[:p, :p] = f11
    rsrc, csrc = _composite(ipiv, p), _composite(jpiv, p)
    out[:p, p:] = out[rsrc, p:]
    out[p:, :p] = out[p:, :][:, csrc]
    if k > 0:
        L11 = np.tril(out[:k, :k], -1) + np.eye(k)
        U11 = np.triu(out[:k, :k])
        out[:k, p:] = np.linalg.solve(L11, out[:k, p:])
        out[k:p, p:] -= out[k:p, :k] @ out[:k, p:]
        out[p:, :k] = np.linalg.solve(U11.T, out[p:, :k].T).T
        out[p:, k:p] -= out[p:, :k] @ out[:k, k:p]
        out[p:, p:] -= out[p:, :k] @ out[:k, p:]
    return k, ipiv, jpiv, out


def _ref_call(name, a, m, n, threads):
    _check(a)
    lda = a.shape[0]
    m = lda if m is None else m
    n = a.shape[1] if n is None else n
    L = ref_lib()
    if threads is not None:
        L.ref_set_threads(int(threads))
    piv = max(min(m, n), 1)
    ipiv = np.zeros(piv, dtype=np.int32)
    jpiv = np.zeros(piv, dtype=np.int32)
    info = ctypes.c_int(-1)
    getattr(L, name)(m, n, a.ctypes.data, lda, _p(ipiv), _p(jpiv), ctypes.byref(info))
    k = min(m, n)
    return ipiv[:k], jpiv[:k], info.value


def ref_getrf(a, m=None, n=None, threads=None):
    """The reference's delayed_getrf (delayed_lu/delayed_dgetrf.cpp:129)."""
    return _ref_call("ref_delayed_getrf", a, m, n, threads)


def ref_getrf_column(a, m=None, n=None, threads=None):
    """The reference's delayed_getrf_column (delayed_lu/delayed_dgetrf_column.cpp:99)."""
    return _ref_call("ref_delayed_getrf_column", a, m, n, threads)


def ref_lapack_getrf(a, m=None, n=None, threads=None):
    """LAPACK dgetrf through the reference's wrapper (delayed_lu/lapack_dgetrf.cpp)."""
    _check(a)
    lda = a.shape[0]
    m = lda if m is None else m
    n = a.shape[1] if n is None else n
    L = ref_lib()
    if threads is not None:
        L.ref_set_threads(int(threads))
    piv = max(min(m, n), 1)
    ipiv = np.zeros(piv, dtype=np.int32)
    info = ctypes.c_int(-1)
    L.ref_lapack_getrf(m, n, a.ctypes.data, lda, _p(ipiv), ctypes.byref(info))
    return ipiv[:min(m, n)], info.value


def residual(orig: np.ndarray, fac: np.ndarray, m: int, n: int, info: int, ipiv, jpiv):
    """Returns (||P A Q - Lbar Ubar||_F, ||A||_F)."""
    _check(orig)
    _check(fac)
    L = oracle_lib()
    k = max(min(m, n), 1)
    ip = np.zeros(k, dtype=np.int32)
    jp = np.zeros(k, dtype=np.int32)
    ip[:len(ipiv)] = ipiv
    jp[:len(jpiv)] = jpiv
    ro = np.zeros(max(m, 1), dtype=np.int32)
    co = np.zeros(max(n, 1), dtype=np.int32)
    work = np.zeros(max(m, 1) * L.oracle_max_threads(), dtype=np.float64)
    out = np.zeros(2, dtype=np.float64)
    L.oracle_residual(m, n, orig.ctypes.data, orig.shape[0], fac.ctypes.data, fac.shape[0],
                      max(info, 0), _p(ip), _p(jp), out.ctypes.data, _p(ro), _p(co),
                      work.ctypes.data)
    return float(out[0]), float(out[1])


def scaled_residual(orig, fac, m, n, info, ipiv, jpiv) -> float:
    """||PAQ - LU||_F / (||A||_F * max(m,n) * u), the acceptance metric (<= 10)."""
    r, an = residual(orig, fac, m, n, info, ipiv, jpiv)
    if an == 0.0:
        return 0.0 if r == 0.0 else float("inf")
    return r / (an * max(m, n) * np.finfo(np.float64).eps / 2)


def ref_binary(name: str):
    """Path of a prebuilt reference-side executable under _ref/ (None when it
    was not built: the reference tree was absent at build time)."""
    p = HERE / "_ref" / name
    return p if p.exists() else None


# ----------------------------------------------- delayed Bunch-Kaufman LDL^T

def sym_matrix(n: int, seed: int, lda: int | None = None, zero_nodes=(), zero_diag: bool = False):
    """A seeded symmetric indefinite test matrix (Fortran, lda >= n): N(0, 1)
    entries mirrored from the lower triangle; `zero_nodes` rows / columns set to
    zero (they can only be delayed); `zero_diag` clears the diagonal (every
    pivot then needs the row test, many become 2x2 blocks)."""
    lda = n if lda is None else lda
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, n))
    a = np.tril(x) + np.tril(x, -1).T
    if zero_diag:
        np.fill_diagonal(a, 0.0)
    for z in zero_nodes:
        a[z, :] = 0.0
        a[:, z] = 0.0
    out = np.zeros((lda, n), order="F")
    out[:n, :n] = a
    return out


def rank8_example(n: int = 4096) -> np.ndarray:
    """The reference's known-answer input (delayed-bunch-kaufman/example.cpp,
    main): zero except a 2x2 block [[0, 2], [2, 0]] at (2, 3) and the diagonal
    6, 5, ..., 1 at positions 4..9 - numerical rank 8, so info = 8."""
    a = np.zeros((n, n), order="F")
    a[3, 2] = a[2, 3] = 2.0
    for k in range(6):
        a[k + 4, k + 4] = float(6 - k)
    return a


def oracle_sytrf(a: np.ndarray, n: int | None = None, nb: int = 64):
    """Factors `a` (Fortran float64, lda = a.shape[0], lower triangle) in place
    by the restatement.  Returns (perm, piv_size, info)."""
    _check(a)
    n = a.shape[1] if n is None else n
    perm = np.zeros(max(n, 1), dtype=np.int32)
    piv = np.zeros(max(n, 1), dtype=np.int32)
    info = oracle_lib().oracle_sytrf(n, a.ctypes.data, a.shape[0], _p(perm), _p(piv), nb)
    return perm[:n], piv[:n], info


def ref_bk_available() -> bool:
    return REF_BK_SO.exists()


def _refbk_lib() -> ctypes.CDLL:
    global _refbk
    if _refbk is None:
        if not REF_BK_SO.exists():
            raise RuntimeError(f"reference CPU build missing: {REF_BK_SO}")
        L = ctypes.CDLL(str(REF_BK_SO))
        for name in ("ref_delayed_sytrf", "ref_delayed_sytrf_blocked", "ref_lapack_sytrf"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _ip(), _ip(), _ip()]
        L.ref_bk_set_threads.restype = None
        L.ref_bk_set_threads.argtypes = [ctypes.c_int]
        _refbk = L
    return _refbk


def ref_sytrf(a: np.ndarray, variant: str = "blocked", threads=None):
    """The reference's delayed_sytrf_blocked (variant "blocked",
    delayed_sytrf_blocked.cpp:141), delayed_sytrf ("unblocked",
    delayed_sytrf.cpp:175) or lapack_sytrf ("lapack", lapack_dsytrf.cpp) on `a`
    in place.  Returns (perm, piv_size, info)."""
    _check(a)
    L = _refbk_lib()
    if threads is not None:
        L.ref_bk_set_threads(int(threads))
    n = a.shape[1]
    perm = np.zeros(max(n, 1), dtype=np.int32)
    piv = np.zeros(max(n, 1), dtype=np.int32)
    info = ctypes.c_int(-1)
    name = {"blocked": "ref_delayed_sytrf_blocked", "unblocked": "ref_delayed_sytrf",
            "lapack": "ref_lapack_sytrf"}[variant]
    getattr(L, name)(n, a.ctypes.data, a.shape[0], _p(perm), _p(piv), ctypes.byref(info))
    return perm[:n], piv[:n], info.value


def ldl_factors(fac: np.ndarray, n: int, piv_size, info: int):
    """Unit-lower L (n x n, identity on the delayed suffix) and block-diagonal
    D (1x1 / 2x2 blocks, then the symmetric delayed Schur complement) from a
    compact factor, as delayed-bunch-kaufman/example.cpp:47-95 reads it."""
    f = np.asarray(fac)[:n, :n]
    piv = np.asarray(piv_size)
    L = np.eye(n)
    D = np.zeros((n, n))
    c = 0
    while c < info:
        if piv[c] == 2:
            L[c + 2:, c] = f[c + 2:, c]
            L[c + 2:, c + 1] = f[c + 2:, c + 1]
            D[c, c], D[c + 1, c + 1] = f[c, c], f[c + 1, c + 1]
            D[c + 1, c] = D[c, c + 1] = f[c + 1, c]
            c += 2
        else:
            L[c + 1:, c] = f[c + 1:, c]
            D[c, c] = f[c, c]
            c += 1
    s = np.tril(f[info:, info:])
    D[info:, info:] = s + np.tril(s, -1).T
    return L, D


def ldl_residual(orig: np.ndarray, fac: np.ndarray, perm, piv_size, info: int) -> float:
    """max |P A P^T - L D L^T| (example.cpp:146-157), A read from orig's lower
    triangle."""
    n = fac.shape[1]
    a = np.tril(np.asarray(orig)[:n, :n])
    a = a + np.tril(a, -1).T
    L, D = ldl_factors(fac, n, piv_size, info)
    p = np.asarray(perm)
    return float(np.abs(a[np.ix_(p, p)] - L @ D @ L.T).max()) if n else 0.0
