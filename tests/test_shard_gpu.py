"""The decomposed solve (grid/multigrid-mpi.h over blocks) against one grid
covering the same domain.

A domain of dims blocks of depth d equals one grid of depth d + log2 dims[0]
whose levels below log2 dims[0] are never visited: poisson () on the blocks
(minlevel 1 of a block) is the single grid's solve with minlevel
1 + log2 dims[0].  With the boundary exchanged after every pass, the blocks
must give the single grid's mgstats (cycles, nrelax, residuals) and
solution bit for bit in FP64; mgstats.sum is a sum in another order."""
import math

import numpy as np
import pytest

from basilisk_b200 import problems
from basilisk_b200.shard import ShardedGrid
from helpers import gpu_grid

pytestmark = pytest.mark.gpu


def sharded(prob, dims, relax):
    k = int(math.log2(dims[0]))
    sg = ShardedGrid(prob["dim"], prob["depth"] - k, dims=dims, periodic=prob["periodic"],
                     relax=relax)
    a = sg.scalar()
    for side, (kind, val) in prob["bc"].items():
        a.bc(side, kind, float(val))
    a.set(np.zeros(prob["b"].shape))
    b = sg.scalar(prob["b"])
    alpha = sg.face_vector(prob["alpha"]) if prob["alpha"] is not None else None
    lam = prob["lambda"]
    if lam is None:
        lam_f = None
    elif np.isscalar(lam):
        lam_f = sg.const_scalar(float(lam))
    else:
        lam_f = sg.scalar(lam)
    return sg, a, b, alpha, lam_f


def compare(prob, dims, relax, tolerance):
    k = int(math.log2(dims[0]))
    g, a, b, alpha, lam = gpu_grid(prob, relax=relax)
    st = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=tolerance, minlevel=1 + k)
    ref = a.get()
    g.close()
    sg, sa, sb, salpha, slam = sharded(prob, dims, relax)
    ss = sg.poisson(sa, sb, alpha=salpha, lambda_=slam, tolerance=tolerance)
    got = sa.get()
    sg.close()
    for key in ("i", "nrelax", "resb", "resa"):
        assert ss[key] == st[key], (key, ss, st)
    assert ss["minlevel"] == 1 and st["minlevel"] == 1 + k
    assert abs(ss["sum"] - st["sum"]) <= 1e-12 * max(1.0, np.abs(prob["b"]).sum())
    np.testing.assert_array_equal(got, ref)
    return ss


@pytest.mark.parametrize("relax", ["rbgs", "jacobi"])
def test_two_phase_2x2_blocks_bit_identical(relax):
    """Dirichlet walls, variable face coefficients (density ratio 1000),
    four blocks of 128^2."""
    compare(problems.two_phase_2d(depth=8, seed=3), (2, 2), relax, 1e-6)


def test_periodic_2x2_blocks_bit_identical():
    """A periodic domain: the blocks' neighbours wrap around."""
    compare(problems.poisson_periodic_2d(depth=8, seed=4), (2, 2), "rbgs", 1e-8)


def test_sixteen_blocks_bit_identical():
    """4 x 4 blocks of 64^2: interior blocks with four neighbours, corner
    ghosts from the diagonal blocks."""
    compare(problems.two_phase_2d(depth=8, seed=6), (4, 4), "rbgs", 1e-6)


def test_mixed_conditions_and_lambda_field_bit_identical():
    """Inhomogeneous Dirichlet on two sides, Neumann on the others (each
    block keeps the condition of the domain's sides it touches), a stored
    lambda field: 2x2 blocks against one grid."""
    import helpers
    rng = np.random.default_rng(21)
    prob = helpers.random_problem(2, 7, rng, bc={0: ("dirichlet", 0.5), 1: ("neumann", -0.25),
                                                 2: ("dirichlet", -1.0), 3: ("neumann", 0.75)},
                                  lam="field")
    compare(prob, (2, 2), "rbgs", 1e-9)


def test_one_block_is_the_grid():
    """dims (1, 1): one block, nothing to exchange (its periodic directions
    are its own), the grid's solve with minlevel 1."""
    compare(problems.poisson_periodic_2d(depth=7, seed=9), (1, 1), "rbgs", 1e-8)


def test_1d_two_blocks_bit_identical():
    """One dimension, two blocks: single-cell ghost slabs."""
    import helpers
    rng = np.random.default_rng(13)
    prob = helpers.random_problem(1, 9, rng, bc={0: ("dirichlet", 1.0), 1: ("dirichlet", -0.5)})
    compare(prob, (2,), "rbgs", 1e-10)


def test_helmholtz_3d_2x2x2_blocks_bit_identical():
    """Periodic 3D Helmholtz (viscosity.h form) on eight blocks of 16^3:
    x slabs, strided y and z slabs."""
    compare(problems.helmholtz_3d(depth=5, seed=7), (2, 2, 2), "rbgs", 1e-8)


def test_two_blocks_rectangular_domain():
    """MPI_Dims_create (2, 2) = (2, 1): a 2:1 domain of two square blocks
    (the reference's rescaled domain, multigrid-mpi.h:115-123), periodic
    along x.  Its solution is symmetric under the shift by one block along
    x when the right-hand side is."""
    n = 64
    rng = np.random.default_rng(8)
    half = rng.standard_normal((n, n))
    half -= half.mean()
    b = np.concatenate([half, half], axis=0)
    sg = ShardedGrid(2, 6, dims=(2, 1), periodic=(0,), relax="rbgs", L0=2.0)
    a = sg.scalar()
    for side in ("top", "bottom"):
        a.bc(side, "dirichlet", 0.0)
    a.set(np.zeros((2 * n, n)))
    bb = sg.scalar(b)
    st = sg.poisson(a, bb, tolerance=1e-8)
    assert st["status"] == 0 and st["resa"] <= 1e-8, st
    sol = a.get()
    sg.close()
    np.testing.assert_array_equal(sol[:n], sol[n:])

