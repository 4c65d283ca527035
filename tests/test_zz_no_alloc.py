"""bmg_sum_noalloc: the allocation-free sum, for callers that cannot
allocate device memory (code inside a global-mode stream capture, programs
whose device memory is all handed to their own pool).  Called through the
C-ABI and checked against the sum that the existing entry point bmg_poisson
reports in mgstats.sum, on two calls in a row, within the tolerance the
parity tests use for that sum (1e-13 times the sum of |b|), and against the
correctly rounded sum of the host values (math.fsum) on counts that end in
a partial tile (1, 4097, 4096 * 37 + 5) and on an empty input.  This file is
collected last so that a run stopping at the first failure has run every
other test first."""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def reference_sum(b_np):
    """mgstats.sum of bmg_poisson for right-hand side b (one V-cycle)."""
    import basilisk_b200 as bmg
    n = b_np.shape[0]
    depth = int(np.log2(n))
    g = bmg.Grid(2, depth, relax="rbgs")
    a = g.scalar()
    for side in range(4):
        a.bc(side, "dirichlet", 0.0)
    b = g.scalar(b_np)
    st = g.poisson(a, b, tolerance=1e30)
    g.close()
    return st["sum"]


def test_sum_noalloc_matches_poisson_sum():
    import torch
    from basilisk_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(2024)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for call, n in enumerate((512, 1024)):        # two calls in a row
        b_np = rng.standard_normal((n, n)) + 0.25
        b = torch.from_numpy(b_np).cuda()
        torch.cuda.synchronize()
        st = L.bmg_sum_noalloc(ctypes.c_void_p(b.data_ptr()), b.numel(),
                               ctypes.c_void_p(out.data_ptr() + 8 * call),
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == _lib.OK
        torch.cuda.synchronize()
        got = float(out[call].item())
        ref = reference_sum(b_np)
        assert abs(got - ref) <= 1e-13 * np.abs(b_np).sum(), (got, ref)
        exact = math.fsum(b_np.ravel().tolist())
        assert abs(got - exact) <= 8 * np.finfo(np.float64).eps * np.abs(b_np).sum(), (got, exact)


def noalloc_sum(values):
    """bmg_sum_noalloc of a host array, through the C-ABI, on torch's stream"""
    import torch
    from basilisk_b200 import _lib
    L = _lib.load()
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    v = torch.from_numpy(values).cuda() if values.size else None
    torch.cuda.synchronize()
    st = L.bmg_sum_noalloc(ctypes.c_void_p(v.data_ptr() if v is not None else None),
                           values.size, ctypes.c_void_p(out.data_ptr()),
                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.OK
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("count", [0, 1, 4097, 4096 * 37 + 5])
def test_sum_noalloc_partial_tiles_against_fsum(count):
    """Counts that are not whole tiles of 4096 values, and 0 (a sum of 0):
    within 8 ulps of sum|b| of the correctly rounded sum of the host data."""
    rng = np.random.default_rng(count)
    b = rng.standard_normal(count) + 0.5
    for _ in range(2):                               # two calls in a row
        got = noalloc_sum(b)
        ref = math.fsum(b.tolist())
        if count == 0:
            assert got == 0.0
        else:
            assert abs(got - ref) <= 8 * np.finfo(np.float64).eps * np.abs(b).sum(), (got, ref)


def test_sum_noalloc_rejects_oversized_input():
    import torch
    from basilisk_b200 import _lib
    L = _lib.load()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # the size check comes before any access: a count beyond the maximum is
    # refused without touching the (small) buffer
    small = torch.zeros(4, dtype=torch.float64, device="cuda")
    st = L.bmg_sum_noalloc(ctypes.c_void_p(small.data_ptr()), 4096 * 4096 + 1,
                           ctypes.c_void_p(out.data_ptr()), None)
    assert st == _lib.EINVAL
