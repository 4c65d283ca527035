"""The CPU oracle against the reference's own golden logs.

The logs (tests/golden/reference_logs.json, collected by
tests/golden/make_golden.py) are the stderr output of the reference's test
programs; tests/golden_drivers.py re-runs those programs on the oracle.
poisson.cref is the multigrid build of test/poisson.c and must match line
for line.  periodic.ref, periodic.3D.ref and poisson1D.ref print converged
errors and must match too.  poisson.ref/poisson.3D.ref/variable.ref were
produced on quadtree/octree grids, whose Gauss-Seidel sweep visits cells in
tree order instead of the multigrid's lexicographic order (poisson.h:284-291
notes that the results depend on it): their final error line must match and
their residual history agree within the spread of the sweep order.
"""
import json
import os

import pytest

import golden_drivers as gd
from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_logs.json")))


def make(dim, depth, origin):
    return oracle.Grid(dim, depth, origin=origin, relax=oracle.RELAX_GS)


PROGRAMS = {
    "poisson_2d": lambda: gd.poisson_program(make, 2),
    "poisson_2d_quadtree": lambda: gd.poisson_program(make, 2),
    "poisson_3d": lambda: gd.poisson_program(make, 3),
    "variable_2d": lambda: gd.variable_program(make),
    "periodic_2d": lambda: gd.periodic_program(make, 2),
    "periodic_3d": lambda: gd.periodic_program(make, 3),
    "poisson_1d": lambda: gd.poisson1d_program(make),
}


@pytest.mark.parametrize("key", ["poisson_2d", "poisson_2d_quadtree", "periodic_2d",
                                 "periodic_3d", "poisson_1d"])
def test_golden_exact(key):
    lines, _ = PROGRAMS[key]()
    assert lines == GOLD[key]["lines"]


@pytest.mark.parametrize("key", ["poisson_3d", "variable_2d"])
def test_golden_tree_order(key):
    lines, _ = PROGRAMS[key]()
    gold = GOLD[key]["lines"]
    assert len(lines) == len(gold)
    assert lines[-1] == gold[-1]          # "# max error ..." identical
    for got, ref in zip(lines[:-1], gold[:-1]):
        gi, gv = got.split()
        ri, rv = ref.split()
        assert gi == ri
        assert abs(float(gv) - float(rv)) <= 0.1 * float(rv), (got, ref)


def test_oracle_jacobi_converges_to_same_solution():
    """The JACOBI branch (poisson.h:293-328) and the default sweep solve the
    same discrete problem."""
    import numpy as np
    from helpers import oracle_grid, random_problem
    rng = np.random.default_rng(5)
    prob = random_problem(2, 5, rng, bc={s: ("dirichlet", 0.0) for s in range(4)})
    sol = []
    for relax in (oracle.RELAX_GS, oracle.RELAX_JACOBI, oracle.RELAX_RBGS):
        g = oracle_grid(prob, relax=relax)
        st = g.poisson(tolerance=1e-12)
        assert st["resa"] <= 1e-12
        sol.append(g.get_a())
    assert np.allclose(sol[0], sol[1], rtol=0, atol=1e-12 * np.abs(sol[0]).max())
    assert np.allclose(sol[0], sol[2], rtol=0, atol=1e-12 * np.abs(sol[0]).max())


def test_oracle_openmp_jacobi_deterministic():
    """Jacobi and red-black sweeps do not depend on the OpenMP thread count."""
    import numpy as np
    from helpers import oracle_grid, random_problem
    rng = np.random.default_rng(6)
    prob = random_problem(2, 7, rng, periodic=(0,), bc={2: ("neumann", 0.0), 3: ("dirichlet", 1.0)})
    for relax in (oracle.RELAX_JACOBI, oracle.RELAX_RBGS):
        out = []
        for threads in (1, 4):
            g = oracle_grid(prob, relax=relax, threads=threads)
            st = g.poisson(tolerance=1e-9)
            out.append((g.get_a(), st["i"], st["resa"]))
        oracle.lib(2).og_set_threads(1)
        assert np.array_equal(out[0][0], out[1][0])
        assert out[0][1:] == out[1][1:]
