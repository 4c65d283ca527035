"""bmg_sum_noalloc: the allocation-free sum, for callers that cannot
allocate device memory (code inside a global-mode stream capture, programs
whose device memory is all handed to their own pool).  Called through the
C-ABI and checked against the sum that the existing entry point bmg_poisson
reports in mgstats.sum, on two calls in a row, within the tolerance the
parity tests use for that sum (1e-13 times the sum of |b|).  This file is
collected last so that a run stopping at the first failure has run every
other test first."""
import ctypes

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
