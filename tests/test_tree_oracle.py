"""The quadtree oracle against the reference's own golden logs.

test/circle.c and test/circle-variable.c run mg_cycle directly on a quadtree
refined inside a circle (depths 7-10) and print every cycle's residual and
the final error; the oracle, driven by the same programs
(tests/golden_drivers.py), must print the same lines."""
import json
import os

import pytest

import golden_drivers as gd
from oracle import tree

HERE = os.path.dirname(os.path.abspath(__file__))
REF = json.load(open(os.path.join(HERE, "golden", "reference_logs.json")))


def make_oracle(relax):
    def make(depth, origin):
        t = tree.Tree(depth, 1.0, origin)
        t.set_relax(relax)
        return t
    return make


@pytest.mark.parametrize("prog,key", [(gd.circle_program, "circle_2d"),
                                      (gd.circle_variable_program, "circle_variable_2d")])
def test_tree_oracle_reproduces_reference_log(prog, key):
    lines, t = prog(make_oracle(tree.RELAX_GS))
    assert lines == REF[key]["lines"]


@pytest.mark.parametrize("relax", [tree.RELAX_JACOBI, tree.RELAX_RBGS])
def test_tree_oracle_other_smoothers_converge_to_same_solution(relax):
    """Jacobi and red-black sweeps change the residual history, not the
    discrete solution: after enough cycles the error lines agree."""
    lines, t = gd.circle_program(make_oracle(relax), depths=(7,), niter=30)
    assert lines[-1] == REF["circle_2d"]["lines"][15]


def test_tree_refinement_is_two_one_balanced():
    """Every leaf's neighbours across a face are at most one level coarser
    or finer (TWO_ONE, grid/tree.h:3), and halo cells exist exactly beside
    refined cells."""
    import numpy as np
    t = tree.Tree(8, 1.0, (-0.5, -0.5))
    t.refine(gd.circle_refinement(8))
    depth = t.depth
    flags = [t.flags(l) for l in range(depth + 1)]
    for l in range(1, depth + 1):
        leaf = (flags[l] & tree.LEAF) != 0
        n = 1 << l
        # a leaf at level l: its parent-level face neighbours must exist (be active)
        pa = (flags[l - 1] & tree.ACTIVE) != 0
        ii, jj = np.nonzero(leaf)
        for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
            pi, pj = (ii + di) // 2, (jj + dj) // 2
            ok = (ii + di >= 0) & (ii + di < n) & (jj + dj >= 0) & (jj + dj < n)
            assert pa[pi[ok], pj[ok]].all()
    assert t.leaves > 0
