"""The CUDA quadtree path against the quadtree oracle and the reference's
golden logs.

The reference's tree programs (test/circle.c, test/circle-variable.c) run
on the library through the C-ABI (tests/golden_drivers.py with the
``GpuTree`` adapter) and on the oracle with the same smoother: every
printed line and every leaf value must agree bit for bit (FP64, the same
evaluation order).  With enough cycles the converged error lines equal the
reference's own."""
import json
import os

import numpy as np
import pytest

import golden_drivers as gd
from helpers import GpuTree
from oracle import tree as ot

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = json.load(open(os.path.join(HERE, "golden", "reference_logs.json")))

RELAX = {"rbgs": ot.RELAX_RBGS, "jacobi": ot.RELAX_JACOBI}


def makers(relax):
    made = {"gpu": [], "cpu": []}

    def gpu(depth, origin):
        t = GpuTree(depth, origin, relax=relax)
        made["gpu"].append(t)
        return t

    def cpu(depth, origin):
        t = ot.Tree(depth, 1.0, origin)
        t.set_relax(RELAX[relax])
        made["cpu"].append(t)
        return t
    return gpu, cpu, made


def leaf_values(t, which):
    out = []
    for l in range(t.depth + 1):
        m = (t.flags(l) & ot.LEAF) != 0
        out.append(t.get_level(which, l)[m])
    return np.concatenate(out)


def test_refinement_matches_oracle():
    for depth in (7, 9):
        g = GpuTree(depth, (-0.5, -0.5))
        c = ot.Tree(depth, 1.0, (-0.5, -0.5))
        cond = gd.circle_refinement(depth)
        assert g.refine(cond) > 0
        c.refine(cond)
        assert g.depth == c.depth and g.leaves == c.leaves
        for l in range(depth + 1):
            np.testing.assert_array_equal(g.flags(l), c.flags(l))
        g.close()


@pytest.mark.parametrize("relax", ["rbgs", "jacobi"])
@pytest.mark.parametrize("prog", [gd.circle_program, gd.circle_variable_program])
def test_tree_programs_bit_identical_to_oracle(prog, relax):
    gpu, cpu, made = makers(relax)
    lines_g, tg = prog(gpu, depths=(7, 8), niter=6)
    lines_c, tc = prog(cpu, depths=(7, 8), niter=6)
    assert lines_g == lines_c
    np.testing.assert_array_equal(leaf_values(tg, ot.A), leaf_values(tc, ot.A))
    np.testing.assert_array_equal(leaf_values(tg, ot.RES), leaf_values(tc, ot.RES))
    for t in made["gpu"]:
        t.close()


@pytest.mark.parametrize("prog,key,niter", [(gd.circle_program, "circle_2d", 30),
                                            (gd.circle_variable_program, "circle_variable_2d", 30)])
def test_tree_converged_error_matches_reference(prog, key, niter):
    """Red-black cycles converge to the reference's discrete solution: the
    error lines of the reference logs (depths 7-10) come out identical."""
    gpu, cpu, made = makers("rbgs")
    lines, t = prog(gpu, niter=niter)
    got = [s for s in lines if s.startswith("max error")]
    want = [s for s in REF[key]["lines"] if s.startswith("max error")]
    assert got == want
    for t in made["gpu"]:
        t.close()


def c4_problem(make, depth, base):
    """The two-phase variable-coefficient problem on a quadtree refined
    within 4 cells of the circle r = 0.25 (graded down to level base)."""
    t = make(depth, (0.0, 0.0))
    t.refine(gd.band_refinement(depth, base))
    gd.two_phase_tree(t, seed=3)
    return t


@pytest.mark.parametrize("relax", ["rbgs", "jacobi"])
def test_tree_poisson_matches_oracle(relax):
    """poisson () on the tree (mg_solve with nrelax adaptation): the same
    statistics and the same solution as the oracle."""
    gpu, cpu, made = makers(relax)
    tg = c4_problem(gpu, 8, 4)
    tc = c4_problem(cpu, 8, 4)
    sg = tg.poisson(tolerance=1e-4, nrelax=4, minlevel=1)
    sc = tc.poisson(tolerance=1e-4, nrelax=4, minlevel=1)
    for k in ("i", "nrelax", "minlevel"):
        assert sg[k] == sc[k], k
    assert sg["resb"] == sc["resb"] and sg["resa"] == sc["resa"]
    assert abs(sg["sum"] - sc["sum"]) <= 1e-12 * max(1.0, abs(sc["sum"]))
    np.testing.assert_array_equal(leaf_values(tg, ot.A), leaf_values(tc, ot.A))
    for t in made["gpu"]:
        t.close()


@pytest.mark.parametrize("relax", ["rbgs", "jacobi"])
def test_tree_interpreter_matches_launch_path(relax):
    """poisson () on the band tree with the iterations run by the schedule
    interpreter (one cluster launch per iteration) and by one launch per
    operation (the tree is built with BMG_NO_TREE_INTERP set): the same
    statistics and leaf values bit for bit, with fewer launches."""
    out = {}
    for interp in (True, False):
        if not interp:
            os.environ["BMG_NO_TREE_INTERP"] = "1"
        try:
            t = GpuTree(9, (0.0, 0.0), relax=relax)
            t.refine(gd.band_refinement(9, 4))
        finally:
            os.environ.pop("BMG_NO_TREE_INTERP", None)
        gd.two_phase_tree(t, seed=11)
        t.g.reset_counters()
        st = t.poisson(tolerance=1e-6, nrelax=4, minlevel=1)
        out[interp] = (st, leaf_values(t, ot.A), t.g.counters())
        t.close()
    (si, ai, ci), (sl, al, cl) = out[True], out[False]
    for k in ("i", "nrelax", "resb", "resa"):
        assert si[k] == sl[k], (k, si, sl)
    np.testing.assert_array_equal(ai, al)
    assert ci["launches"] < cl["launches"], (ci, cl)


def test_tree_mixed_form_against_the_oracle():
    """The mixed form on the band tree (FP32 cycles inside FP64 iterative
    refinement): it reaches the tolerance, its error against the tree
    oracle driven to 1e-9 (124 cycles) is no worse than a small multiple of
    the FP64 form's at the same tolerance (1e-6), and driven on to 1e-9 it
    is close to the oracle's solution."""
    import basilisk_b200 as bmg
    depth, base = 8, 4
    ot.set_niter(nitermax=400)
    try:
        tc = c4_problem(lambda d, o: _cpu_rbgs(d, o), depth, base)
        sc = tc.poisson(tolerance=1e-9, nrelax=4, minlevel=1)
    finally:
        ot.set_niter(nitermax=100)
    assert sc["resa"] <= 1e-9, sc
    ref = leaf_values(tc, ot.A)
    errs = {}
    for prec in ("fp64", "mixed"):
        tg = c4_problem(lambda d, o: GpuTree(d, o, relax="rbgs", precision=prec), depth, base)
        st = tg.poisson(tolerance=1e-6, nrelax=4, minlevel=1)
        assert st["resa"] <= 1e-6, (prec, st)
        errs[prec] = float(np.abs(leaf_values(tg, ot.A) - ref).max() / np.abs(ref).max())
        if prec == "mixed":
            bmg.set_niter(nitermax=400)
            try:
                st = tg.poisson(tolerance=1e-9, nrelax=4, minlevel=1)
            finally:
                bmg.set_niter(nitermax=100)
            assert st["resa"] <= 1e-9, st
            errs["mixed_1e-9"] = float(np.abs(leaf_values(tg, ot.A) - ref).max()
                                       / np.abs(ref).max())
        tg.close()
    print("tree errors against the oracle:", errs)
    assert errs["mixed"] <= 4 * errs["fp64"] + 1e-12, errs
    assert errs["mixed_1e-9"] <= 1e-6, errs


def test_tree_mixed_form_jacobi_reaches_the_tolerance():
    """The mixed form with the reference's weighted-Jacobi smoother on the
    tree (the interpreter's FP32 Jacobi temporary): it reaches the
    tolerance (1e-4: the reference's Jacobi branch stalls near 2e-5 on this
    problem), and both forms' solutions agree to the accuracy that residual
    pins."""
    depth, base = 8, 4
    sols = {}
    for prec in ("fp64", "mixed"):
        tg = c4_problem(lambda d, o: GpuTree(d, o, relax="jacobi", precision=prec), depth, base)
        st = tg.poisson(tolerance=1e-4, nrelax=4, minlevel=1)
        assert st["resa"] <= 1e-4, (prec, st)
        sols[prec] = leaf_values(tg, ot.A)
        tg.close()
    rel = float(np.abs(sols["mixed"] - sols["fp64"]).max() / np.abs(sols["fp64"]).max())
    assert rel <= 1e-3, rel


def test_tree_mixed_form_needs_the_interpreter():
    """A tree built without the schedule interpreter (BMG_NO_TREE_INTERP set
    when it is refined) solves in FP64, and refuses the mixed form with
    BMG_EUNSUPPORTED instead of computing anything else."""
    import basilisk_b200 as bmg
    os.environ["BMG_NO_TREE_INTERP"] = "1"
    try:
        t = GpuTree(7, (0.0, 0.0), relax="rbgs", precision="mixed")
        t.refine(gd.band_refinement(7, 4))
    finally:
        os.environ.pop("BMG_NO_TREE_INTERP", None)
    gd.two_phase_tree(t, seed=2)
    st = t.g.poisson(t.f[ot.A], t.f[ot.B], alpha=t.alpha, tolerance=1e-6, check_status=False)
    assert st["status"] == bmg._lib.EUNSUPPORTED, st
    t.g.set_precision("fp64")
    st = t.g.poisson(t.f[ot.A], t.f[ot.B], alpha=t.alpha, tolerance=1e-6, check_status=False)
    assert st["status"] == 0 and st["resa"] <= 1e-6, st
    t.close()


def _cpu_rbgs(depth, origin):
    t = ot.Tree(depth, 1.0, origin)
    t.set_relax(ot.RELAX_RBGS)
    return t
