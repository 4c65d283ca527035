"""The synthetic workloads (basilisk_b200/problems.py): shapes, seeding and
the recipes the benchmark configurations state (two-phase alpha = 1/rho of
the face-averaged volume fraction with density ratio 1000, periodic face
vectors with face n the image of face 0, the quadtree band)."""
import math

import numpy as np

from basilisk_b200 import problems


def test_two_phase_2d_recipe():
    p = problems.two_phase_2d(depth=6, seed=1)
    n = 64
    assert p["b"].shape == (n, n) and p["dim"] == 2 and p["periodic"] == ()
    assert all(p["bc"][s] == ("dirichlet", 0.0) for s in range(4))
    ax, ay = p["alpha"]
    assert ax.shape == (n + 1, n) and ay.shape == (n, n + 1)
    # alpha = 1/rho with rho between 1 (inside the circle) and 1000 (outside)
    for a in (ax, ay):
        assert a.min() >= 1.0 / 1000.0 - 1e-15 and a.max() <= 1.0 + 1e-15
    # centre: the light phase (the tanh profile of width 2 Delta leaves a
    # 1e-4 trace of the heavy one eight cells from the interface)
    assert math.isclose(ax[n // 2, n // 2], 1.0, rel_tol=1e-3)
    assert math.isclose(ax[0, 0], 1e-3, rel_tol=1e-6)                # corner: heavy phase
    # the face values are symmetric under the exchange of x and y
    np.testing.assert_allclose(ax, ay.T, rtol=0, atol=1e-15)
    # seeded: the same seed gives the same right-hand side, another seed not
    assert np.array_equal(p["b"], problems.two_phase_2d(depth=6, seed=1)["b"])
    assert not np.array_equal(p["b"], problems.two_phase_2d(depth=6, seed=2)["b"])


def test_random_field_faces_are_periodic():
    p = problems.random_field_2d(depth=5, seed=3, instance=2)
    n = 32
    kx, ky = p["alpha"]
    assert kx.shape == (n + 1, n) and ky.shape == (n, n + 1)
    np.testing.assert_array_equal(kx[n], kx[0])          # face n is the image of face 0
    np.testing.assert_array_equal(ky[:, n], ky[:, 0])
    k = p["kappa"]
    np.testing.assert_allclose(kx[1:n], np.exp((k[:-1] + k[1:]) / 2.0), rtol=1e-15)
    # instances of one seed differ
    q = problems.random_field_2d(depth=5, seed=3, instance=3)
    assert not np.array_equal(p["kappa"], q["kappa"])


def test_helmholtz_3d_recipe():
    p = problems.helmholtz_3d(depth=3, seed=2)
    n = 8
    assert p["periodic"] == (0, 1, 2) and p["lambda"] == -1000.0 and p["tolerance"] == 1e-8
    assert [a.shape for a in p["alpha"]] == [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)]
    assert all(np.all(a == 1e-2) for a in p["alpha"])
    # four weighted-Jacobi smoothing sweeps of white noise reduce its variance
    raw = np.random.default_rng(2).standard_normal((n, n, n))
    assert p["b"].std() < raw.std()


def test_band_refinement():
    cond = problems.band_refinement(depth=9, base=5)
    assert cond(4, 0.0, 0.0)                       # every cell below the base level
    assert not cond(9, 0.75, 0.5)                  # never past the depth
    assert cond(7, 0.75, 0.5)                      # on the circle r = 0.25
    assert not cond(7, 0.5, 0.5)                   # far from it


def test_two_phase_tree_configuration():
    """The quadtree workload (two_phase_tree): every cell below level 5 and a
    band of four cells of each level around r = 0.25 refined up to level 11,
    2:1 balanced, gives 77,068 leaves on levels 5 to 11 (the tree oracle's
    refine, tree-common.h:308-326)."""
    from oracle import tree as otree
    t = otree.Tree(11)
    t.refine(problems.band_refinement(11, 5))
    assert t.depth == 11 and t.leaves == 77068
    levels = [l for l in range(12) if ((t.flags(l) & otree.LEAF) != 0).any()]
    assert levels == list(range(5, 12))
