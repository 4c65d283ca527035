"""The fused 3D red-black sweep (k_relax3d_rb: a whole sweep in one launch,
planes streamed through shared memory) against the two one-pass launches
it replaces (the grid is created with BMG_FUSED3D set for the fused one).  The
fused kernel evaluates relax_value's expression in the same order, so both
paths give the same mgstats and solution bit for bit, in FP64 and in the
mixed form's FP32 cycles (and the one-pass path is bit-compared with the
oracle by the 3D cases of test_parity_gpu.py and test_full_size_parity.py)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solve(prob, fused, precision, tol):
    from helpers import gpu_grid
    if fused:
        os.environ["BMG_FUSED3D"] = "1"
    try:
        g, a, b, alpha, lam = gpu_grid(prob, relax="rbgs", precision=precision)
    finally:
        os.environ.pop("BMG_FUSED3D", None)
    g.reset_counters()
    st = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=tol)
    sol, c = a.get(), g.counters()
    g.close()
    return st, sol, c


def cases():
    import helpers
    from basilisk_b200 import problems
    rng = np.random.default_rng(31)
    return {
        "helmholtz_periodic_64": problems.helmholtz_3d(depth=6, seed=3),
        "dirichlet_neumann_lambda_field_32": helpers.random_problem(
            3, 5, rng, bc={0: ("dirichlet", 0.25), 1: ("neumann", 0.5), 2: ("dirichlet", 0.0),
                           3: ("dirichlet", -1.0), 4: ("neumann", 0.0), 5: ("dirichlet", 0.0)},
            lam="field"),
        "periodic_y_64": helpers.random_problem(
            3, 6, rng, periodic=(1,), bc={0: ("dirichlet", 0.0), 1: ("dirichlet", 0.0),
                                          4: ("neumann", 0.0), 5: ("neumann", 0.0)}, lam=-3.0),
        "neumann_16": helpers.random_problem(
            3, 4, rng, bc={s: ("neumann", 0.0) for s in range(6)}, lam=-1.0),
    }


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["helmholtz_periodic_64", "dirichlet_neumann_lambda_field_32",
                                  "periodic_y_64", "neumann_16"])
def test_fused_sweep_matches_two_passes(name, precision):
    prob = cases()[name]
    sf, af, cf = solve(prob, True, precision, 1e-9)
    so, ao, co = solve(prob, False, precision, 1e-9)
    for k in ("i", "nrelax", "resb", "resa"):
        assert sf[k] == so[k], (k, sf, so)
    assert sf["resa"] <= 1e-9
    np.testing.assert_array_equal(af, ao)
    # one launch per sweep instead of two on the fused levels (a 16^3
    # mixed-form hierarchy lies entirely in the single-CTA bottom solve)
    assert cf["launches"] <= co["launches"], (cf, co)
    if prob["depth"] >= 5:
        assert cf["launches"] < co["launches"], (cf, co)
