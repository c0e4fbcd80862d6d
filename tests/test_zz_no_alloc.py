"""GPU test of dp_getrf_device_noalloc, the entry point for callers that
cannot allocate device memory during a call (a memory manager that owns the
whole pool, a fixed HBM budget, an allocator other than the CUDA runtime's).

It is called twice in a row on the same input through the C ABI and each
result is checked against dp_getrf_device: identical pivot records and info,
factors equal within the tests' residual bound (scaled residual <= 10, the
same bound as the parity tests), and the scaled residual itself <= 10.  The
allocation-free path solves the outer blocks' triangular systems by
substitution (it has no room for their inverses), so its factors are
compared with dp_getrf_device in that mode (dp_block_solve(2)); its records
must also equal those of the default (by inverse) mode.
Inputs beyond its fixed scratch are rejected before any device work.

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test; it also passes alone.
"""
import numpy as np
import pytest

import golden_cases as gc

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _factor(fn, a, m, n):
    torch = _torch()
    d = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    k = min(m, n)
    ipiv = np.full(k, -5, dtype=np.int32)
    jpiv = np.full(k, -5, dtype=np.int32)
    st, info = fn(m, n, d, a.shape[0], ipiv, jpiv)
    torch.cuda.synchronize()
    return st, info, ipiv, jpiv, np.asfortranarray(d.cpu().numpy().T)


@pytest.mark.parametrize("name", ["config1_n1024", "square_517_lda520", "tall_300x200",
                                  "ref_far_pivot_70"])
def test_noalloc_matches_allocating_entry_point_twice(built, name):
    import delayed_pivoting as dp
    import oracle as orc

    a, case = gc.load(name)
    m, n = case["m"], case["n"]
    st1, info1, ip1, jp1, _ = _factor(dp.delayed_getrf_cuda_device, a, m, n)
    prev = dp.block_solve(2)
    try:
        st0, info0, ip0, jp0, f0 = _factor(dp.delayed_getrf_cuda_device, a, m, n)
    finally:
        dp.block_solve(prev)
    assert st0 == st1 == dp.SUCCESS and info0 == info1
    np.testing.assert_array_equal(ip0, ip1)
    np.testing.assert_array_equal(jp0, jp1)
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        st, info, ip, jp, f = _factor(dp.getrf_device_noalloc, a, m, n)
        assert st == dp.SUCCESS
        assert info == info0 == case["info"]
        np.testing.assert_array_equal(ip, ip0)
        np.testing.assert_array_equal(jp, jp0)
        res = orc.scaled_residual(a, f, m, n, info, ip, jp)
        assert res <= 10.0
        scale = max(1.0, float(np.abs(a).max()))
        assert np.abs(f - f0).max() <= 10.0 * max(m, n) * np.finfo(np.float64).eps * scale


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import delayed_pivoting as dp

    _torch()
    n = 40000  # more than the 32768 pivots the fixed scratch holds
    ipiv = np.zeros(n, dtype=np.int32)
    jpiv = np.zeros(n, dtype=np.int32)
    # rejected before the (never dereferenced) matrix pointer is touched
    assert dp.getrf_device_noalloc(n, n, 0x1000, n, ipiv, jpiv) == (dp.INVALID_ARGUMENT, -1)
