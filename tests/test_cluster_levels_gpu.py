"""The cluster level kernel of the mixed form (k_level_cluster: all nrelax
sweeps of a 128^2 or 256^2 FP32 level in one launch of one thread-block
cluster, halos exchanged through distributed shared memory, the
prolongation fused in) against the launch-per-four-sweeps tile path it
replaces (the grid is created with BMG_NO_CLUSTER set for that one).  Both are the FP32 smoothing of the same
operator inside the FP64 refinement, so they reach the tolerance in about
the same number of cycles and their solutions agree to the solve's
accuracy; the FP64 oracle at 1e-12 bounds both."""
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


def solve_mixed(prob, persist, tol):
    from helpers import gpu_grid
    if not persist:
        os.environ["BMG_NO_CLUSTER"] = "1"
    try:
        g, a, b, alpha, lam = gpu_grid(prob, relax="rbgs", precision="mixed")
    finally:
        os.environ.pop("BMG_NO_CLUSTER", None)
    st = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=tol)
    sol, c = a.get(), g.counters()
    g.close()
    return st, sol, c


def oracle_solution(prob):
    from helpers import oracle_grid
    o = oracle_grid(prob, relax=oracle.RELAX_RBGS, threads=os.cpu_count() or 1)
    o.poisson(tolerance=1e-12)
    return o.get_a()


def cases():
    import helpers
    from basilisk_b200 import problems
    rng = np.random.default_rng(77)
    return {
        "two_phase_512": problems.two_phase_2d(depth=9, seed=4),
        "periodic_256": problems.poisson_periodic_2d(depth=8, seed=5),
        "neumann_lambda_field_512": helpers.random_problem(
            2, 9, rng, bc={s: ("neumann", 0.0) for s in range(4)}, lam="field"),
        "mixed_bc_128": helpers.random_problem(
            2, 7, rng, periodic=(1,), bc={0: ("dirichlet", 0.5), 1: ("neumann", -0.25)}),
    }


@pytest.mark.parametrize("name", ["two_phase_512", "periodic_256", "neumann_lambda_field_512",
                                  "mixed_bc_128"])
def test_cluster_levels_match_tile_path(name):
    prob = cases()[name]
    tol = 1e-9
    sp, ap, cp = solve_mixed(prob, True, tol)
    st, at, ct = solve_mixed(prob, False, tol)
    assert sp["resa"] <= tol and st["resa"] <= tol, (sp, st)
    # two FP32 trajectories of the refinement: a couple of cycles apart at most
    assert abs(sp["i"] - st["i"]) <= max(2, 0.05 * st["i"]), (sp, st)
    ref = oracle_solution(prob)
    if not any(k == "dirichlet" for k, _ in prob["bc"].values()) and prob["lambda"] is None:
        ap, at, ref = ap - ap.mean(), at - at.mean(), ref - ref.mean()
    scale = np.abs(ref).max()
    ep, et = np.abs(ap - ref).max() / scale, np.abs(at - ref).max() / scale
    assert ep <= max(4 * et, 1e-9) and et <= max(4 * ep, 1e-9), (ep, et)
    # one launch per middle level instead of nrelax/4 + 1 tile launches
    # (at nrelax = 4 the 64^2 level's own launch can make it one more)
    if sp["nrelax"] >= 8 and st["nrelax"] >= 8:
        assert cp["launches"] / cp["cycles"] < ct["launches"] / ct["cycles"], (cp, ct)


@pytest.mark.parametrize("depth", [7, 8])
def test_cluster_level_finest(depth):
    """A grid whose finest level is a cluster level (128^2, 256^2): the
    level's final iterate feeds the correction a += da."""
    from basilisk_b200 import problems
    prob = problems.two_phase_2d(depth=depth, seed=9)
    sp, ap, _ = solve_mixed(prob, True, 1e-6)
    st, at, _ = solve_mixed(prob, False, 1e-6)
    assert sp["resa"] <= 1e-6 and abs(sp["i"] - st["i"]) <= 2, (sp, st)
    assert np.abs(ap - at).max() <= 1e-3 * np.abs(at).max()


def solve_fp64(prob, cluster, tol):
    from helpers import gpu_grid
    if not cluster:
        os.environ["BMG_NO_CLUSTER"] = "1"
    try:
        g, a, b, alpha, lam = gpu_grid(prob, relax="rbgs")
    finally:
        os.environ.pop("BMG_NO_CLUSTER", None)
    st = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=tol)
    sol = a.get()
    g.close()
    return st, sol


@pytest.mark.parametrize("name", ["two_phase_512", "periodic_256", "neumann_lambda_field_512",
                                  "mixed_bc_128"])
def test_fp64_cluster_levels_bit_identical(name):
    """The plain FP64 form's cluster kernel (64^2 and 128^2 levels, relax_value's
    order with the IEEE division) gives the tile / single-CTA path's solve and
    the oracle's bit for bit."""
    from helpers import oracle_grid
    prob = cases()[name]
    sc, ac = solve_fp64(prob, True, 1e-8)
    st, at = solve_fp64(prob, False, 1e-8)
    for k in ("i", "nrelax", "resb", "resa"):
        assert sc[k] == st[k], (k, sc, st)
    assert np.array_equal(ac, at)
    o = oracle_grid(prob, relax=oracle.RELAX_RBGS, threads=os.cpu_count() or 1)
    so = o.poisson(tolerance=1e-8)
    assert so["i"] == sc["i"] and so["resa"] == sc["resa"], (so, sc)
    assert np.array_equal(o.get_a(), ac)
