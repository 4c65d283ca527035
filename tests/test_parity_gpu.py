"""Parity of the CUDA path (through the C-ABI) with the CPU oracle.

The oracle restates the reference's algorithm (oracle/mg_oracle.c); both are
fed the same seeded inputs.  The weighted-Jacobi smoother (the reference's
-DJACOBI branch) and the red-black smoother (the oracle's extension of the
same name) are order-independent, and the library is compiled without FMA
contraction, so their FP64 results must be bit-identical: solution,
residuals, iteration count and nrelax.  mgstats.sum is a reduction whose
order differs (serial on the CPU, a fixed two-stage tree on the GPU): equal
to 1e-12 relative.
"""
import numpy as np
import pytest

from helpers import gpu_grid, oracle_grid, random_problem
from oracle import oracle

pytestmark = pytest.mark.gpu

RELAX = {"jacobi": oracle.RELAX_JACOBI, "rbgs": oracle.RELAX_RBGS}


def solve_both(prob, relax, tolerance=1e-6, nrelax=4, minlevel=0, graphs=True):
    og = oracle_grid(prob, relax=RELAX[relax])
    ost = og.poisson(tolerance=tolerance, nrelax=nrelax, minlevel=minlevel)
    g, a, b, alpha, lam = gpu_grid(prob, relax=relax, graphs=graphs)
    gst = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=tolerance, nrelax=nrelax,
                    minlevel=minlevel)
    return og, ost, g, a, gst


def assert_same(ost, gst, oa, ga, b=None):
    assert gst["i"] == ost["i"]
    assert gst["nrelax"] == ost["nrelax"]
    assert gst["minlevel"] == ost["minlevel"]
    assert gst["resb"] == ost["resb"]
    assert gst["resa"] == ost["resa"]
    # the sum's rounding depends on the summation order: bound it by eps*sum|b|
    scale = np.abs(b).sum() if b is not None else max(1.0, abs(ost["sum"]))
    assert abs(gst["sum"] - ost["sum"]) <= 1e-13 * scale + 1e-300
    assert np.array_equal(ga, oa), np.abs(ga - oa).max()


CASES = [
    # dim, depth, periodic, bc, alpha, lambda
    (2, 6, (), {s: ("dirichlet", 0.0) for s in range(4)}, "field", None),
    (2, 7, (0, 1), {}, 1.0, None),
    (2, 5, (0,), {2: ("neumann", 0.5), 3: ("dirichlet", 1.0)}, "field", "field"),
    (2, 6, (1,), {0: ("dirichlet", -1.0), 1: ("neumann", 0.0)}, "field", -3.0),
    (2, 4, (), {0: ("neumann", 0.0), 1: ("neumann", 0.0), 2: ("neumann", 0.0),
                3: ("dirichlet", 0.0)}, 2.5, None),
    (1, 8, (), {0: ("dirichlet", 1.0), 1: ("dirichlet", -2.0)}, "field", None),
    (1, 6, (0,), {}, "field", -1.0),
    (3, 4, (0, 1, 2), {}, "field", -50.0),
    (3, 5, (), {s: ("dirichlet", 0.0) for s in range(6)}, "field", None),
    (3, 4, (2,), {0: ("dirichlet", 0.3), 1: ("neumann", 0.0), 2: ("neumann", 1.0),
                  3: ("dirichlet", 0.0)}, 0.7, "field"),
]


@pytest.mark.parametrize("relax", ["jacobi", "rbgs"])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_poisson_bit_exact(case, relax):
    dim, depth, per, bc, al, lam = CASES[case]
    rng = np.random.default_rng(100 + case)
    prob = random_problem(dim, depth, rng, periodic=per, bc=bc, alpha=al, lam=lam, a0=True)
    og, ost, g, a, gst = solve_both(prob, relax, tolerance=1e-7)
    assert_same(ost, gst, og.get_a(), a.get(), prob["b"])


@pytest.mark.parametrize("L0", [1.0, 3.0, 0.25])
def test_domain_size_bit_exact(L0):
    """Delta = L0/2^l: a power of two (the residual scales by 1/Delta
    exactly) or not (it divides, in the reference's order); both
    bit-identical to the oracle."""
    rng = np.random.default_rng(17)
    prob = random_problem(2, 6, rng, bc={s: ("dirichlet", 0.0) for s in range(4)}, alpha="field")
    og = oracle_grid(prob, relax=RELAX["rbgs"], L0=L0)
    ost = og.poisson(tolerance=1e-7)
    g, a, b, alpha, lam = gpu_grid(prob, relax="rbgs", L0=L0)
    gst = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=1e-7)
    assert_same(ost, gst, og.get_a(), a.get(), prob["b"])


LARGE = [
    # larger 2D levels: several shared-memory tiles per level, tile edges,
    # lambda staged in shared memory, periodic halos wrapping across tiles
    (2, 9, (), {s: ("dirichlet", 0.0) for s in range(4)}, "field", None),
    (2, 9, (0, 1), {}, "field", -2.0),
    (2, 8, (1,), {0: ("dirichlet", 1.0), 1: ("neumann", -0.5)}, "field", "field"),
    (2, 10, (0,), {2: ("neumann", 0.0), 3: ("dirichlet", 0.0)}, 1.0, None),
    # stored lambda on a 512^2 level (its first tile launch stages the
    # prolongation and lambda), periodic across one axis
    (2, 9, (1,), {0: ("dirichlet", 0.5), 1: ("neumann", 0.25)}, "field", "field"),
]


@pytest.mark.parametrize("case", range(len(LARGE)))
def test_rbgs_large_levels_bit_exact(case):
    dim, depth, per, bc, al, lam = LARGE[case]
    rng = np.random.default_rng(300 + case)
    prob = random_problem(dim, depth, rng, periodic=per, bc=bc, alpha=al, lam=lam)
    og, ost, g, a, gst = solve_both(prob, "rbgs", tolerance=1e-7)
    assert_same(ost, gst, og.get_a(), a.get(), prob["b"])


@pytest.mark.parametrize("case", range(len(LARGE)))
def test_mixed_large_levels(case):
    """The mixed form on the same large levels (FP32 tiles with
    register-resident weights on levels of 512^2 and more: domain edges,
    periodic wrap, constant and stored alpha and lambda): it converges to
    the tolerance in about the oracle's number of cycles, to the oracle's
    solution within the tolerance-implied bound."""
    dim, depth, per, bc, al, lam = LARGE[case]
    rng = np.random.default_rng(300 + case)
    prob = random_problem(dim, depth, rng, periodic=per, bc=bc, alpha=al, lam=lam)
    og = oracle_grid(prob, relax=RELAX["rbgs"])
    ost = og.poisson(tolerance=1e-7)
    g, a, b, alpha, lamf = gpu_grid(prob, relax="rbgs", precision="mixed")
    gst = g.poisson(a, b, alpha=alpha, lambda_=lamf, tolerance=1e-7)
    assert gst["resa"] <= 1e-7, gst
    assert gst["i"] <= 1.25 * ost["i"] + 1, (gst, ost)
    ref, got = og.get_a(), a.get()
    if per and lam is None:          # defined up to a constant
        ref, got = ref - ref.mean(), got - got.mean()
    assert np.abs(got - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_phase_rbgs(precision):
    """The two-phase recipe at 256^2 on the red-black path: bit-identical in
    FP64; the mixed form within the tolerance-implied bound of the oracle."""
    from basilisk_b200 import problems
    prob = problems.two_phase_2d(depth=8, seed=12)
    og = oracle_grid(prob, relax=oracle.RELAX_RBGS)
    ost = og.poisson(tolerance=1e-6)
    g, a, b, alpha, lam = gpu_grid(prob, relax="rbgs", precision=precision)
    gst = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=1e-6)
    if precision == "fp64":
        assert_same(ost, gst, og.get_a(), a.get(), prob["b"])
    else:
        assert gst["resa"] <= 1e-6
        # FP32 smoothing changes the trajectory, not the convergence rate
        assert gst["i"] <= 1.2*ost["i"]
        ref = og.get_a()
        assert np.abs(a.get() - ref).max() <= 1e-3 * np.abs(ref).max()


@pytest.mark.parametrize("relax", ["jacobi", "rbgs"])
def test_per_face_boundary_values(relax):
    """Dirichlet / Neumann data given per boundary face (a[left] =
    dirichlet(f(y)) in the reference)."""
    rng = np.random.default_rng(7)
    n = 32
    bc = {0: ("dirichlet", rng.standard_normal(n)), 1: ("neumann", rng.standard_normal(n)),
          2: ("dirichlet", rng.standard_normal(n)), 3: ("dirichlet", rng.standard_normal(n))}
    prob = random_problem(2, 5, rng, bc=bc, alpha="field")
    og, ost, g, a, gst = solve_both(prob, relax, tolerance=1e-8)
    assert_same(ost, gst, og.get_a(), a.get(), prob["b"])


@pytest.mark.parametrize("graphs", [True, False])
def test_two_phase_config_small(graphs):
    """The two-phase recipe (density ratio 1000, Dirichlet 0) at 128^2: nrelax
    adapts upward; trajectories identical."""
    from basilisk_b200 import problems
    prob = problems.two_phase_2d(depth=7, seed=11)
    og = oracle_grid(prob, relax=RELAX["jacobi"])
    ost = og.poisson(tolerance=1e-6, nrelax=4)
    g, a, b, alpha, lam = gpu_grid(prob, relax="jacobi", graphs=graphs)
    g.set_timing(True)       # per-cycle CUDA events, captured or plain
    gst = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=1e-6, nrelax=4)
    assert_same(ost, gst, og.get_a(), a.get(), prob["b"])
    assert ost["nrelax"] > 4
    c = g.counters()
    assert c["cycles"] == gst["i"] and c["cycle_ms"] > 0 and c["relax_ms"] > 0


def test_periodic_gaussians_128():
    """The 128^2 periodic Gaussian-bump Poisson problem, solved end to end."""
    from basilisk_b200 import problems
    prob = problems.poisson_periodic_2d(depth=7, seed=0)
    for relax in ("jacobi", "rbgs"):
        og, ost, g, a, gst = solve_both(prob, relax, tolerance=1e-6)
        assert_same(ost, gst, og.get_a(), a.get(), prob["b"])
        assert gst["resa"] <= 1e-6


@pytest.mark.parametrize("minlevel", [0, 1, 3])
def test_minlevel(minlevel):
    rng = np.random.default_rng(8)
    prob = random_problem(2, 6, rng, bc={s: ("dirichlet", 0.0) for s in range(4)})
    og, ost, g, a, gst = solve_both(prob, "jacobi", tolerance=1e-8, minlevel=minlevel)
    assert_same(ost, gst, og.get_a(), a.get(), prob["b"])
    assert gst["minlevel"] == max(1, minlevel)


@pytest.mark.parametrize("depth", [0, 1, 2])
@pytest.mark.parametrize("per", [(), (0, 1), (0,)])
def test_tiny_grids(depth, per):
    """Levels 0-2, including the level-0 periodic rule (multigrid.h:655-664)."""
    rng = np.random.default_rng(9 + depth)
    bc = {} if len(per) == 2 else {s: ("dirichlet", 0.5) for s in range(4) if s // 2 not in per}
    prob = random_problem(2, depth, rng, periodic=per, bc=bc, alpha="field", lam=-1.0)
    og = oracle_grid(prob, relax=oracle.RELAX_JACOBI)
    og.restrict_coefficients()
    g, a, b, alpha, lam = gpu_grid(prob, relax="jacobi")
    res_g = g.scalar()
    dp = g.scalar()
    for side in range(4):
        if side // 2 not in per:
            dp.bc(side, "dirichlet", 0.0)
    g.restriction([alpha])
    r0 = og.residual()
    r1 = g.residual(a, b, res_g, alpha=alpha, lambda_=lam)
    assert r0 == r1
    for _ in range(3):
        og.mg_cycle(3, 0, depth)
        g.mg_cycle(a, res_g, dp, 3, 0, depth, alpha=alpha, lambda_=lam)
        assert og.residual() == g.residual(a, b, res_g, alpha=alpha, lambda_=lam)
    assert np.array_equal(og.get_a(), a.get())


# ---- the reference's own test programs on the GPU ----------------------

class GPUDriverGrid:
    """The interface tests/golden_drivers.py expects, on the CUDA library."""

    def __init__(self, dim, depth, origin, relax="rbgs"):
        import basilisk_b200 as bmg
        self.ref = oracle.Grid(dim, depth, origin=origin)   # geometry helpers only
        self.dim, self.depth, self.n = dim, depth, 1 << depth
        self.g = bmg.Grid(dim, depth, origin=origin, relax=relax)
        self.a, self.b, self.res, self.dp = (self.g.scalar(), self.g.scalar(),
                                              self.g.scalar(), self.g.scalar())
        self.alpha = None
        self.lam = None
        self.bcs = []

    delta = property(lambda self: self.ref.delta)
    centers = property(lambda self: self.ref.centers)
    face_centers = property(lambda self: self.ref.face_centers)
    boundary_points = property(lambda self: self.ref.boundary_points)

    def set_periodic(self, d):
        self.g.periodic(2 * d)

    def set_bc(self, side, kind, value=0.0, values=None):
        k = "dirichlet" if kind == oracle.DIRICHLET else "neumann"
        self.a.bc(side, k, value, values=values)
        self.dp.bc(side, k, 0.0)

    def set_a(self, v):
        self.a.set(v)

    def set_b(self, v):
        self.b.set(v)

    def get_a(self):
        return self.a.get()

    def set_alpha(self, comps):
        self.alpha = self.g.face_vector(comps)

    def set_alpha_const(self, v):
        self.alpha = self.g.const_face_vector(v) if v != 1.0 else None

    def set_lambda_const(self, v):
        self.lam = self.g.const_scalar(v) if v != 0.0 else None

    def restrict_coefficients(self):
        if self.alpha is not None and self.alpha.const is None:
            self.g.restriction([self.alpha])

    def residual(self):
        return self.g.residual(self.a, self.b, self.res, alpha=self.alpha, lambda_=self.lam)

    def mg_cycle(self, nrelax, minlevel, maxlevel):
        self.g.mg_cycle(self.a, self.res, self.dp, nrelax, minlevel, maxlevel,
                        alpha=self.alpha, lambda_=self.lam)

    def set_tolerance_global(self, t):
        import basilisk_b200 as bmg
        bmg.set_tolerance(t)

    def poisson(self):
        return self.g.poisson(self.a, self.b, alpha=self.alpha, lambda_=self.lam)


def gpu_make(relax):
    def make(dim, depth, origin):
        return GPUDriverGrid(dim, depth, origin, relax=relax)
    return make


@pytest.mark.parametrize("relax", ["rbgs", "jacobi"])
def test_golden_programs_on_gpu_match_oracle(relax):
    """test/poisson.c, variable.c, periodic.c and poisson1D.c on the GPU
    print exactly what the oracle prints with the same smoother."""
    import golden_drivers as gd

    def omake(dim, depth, origin):
        return oracle.Grid(dim, depth, origin=origin, relax=RELAX[relax])

    for prog in (lambda m: gd.poisson_program(m, 2), lambda m: gd.poisson_program(m, 3),
                 gd.variable_program, lambda m: gd.periodic_program(m, 2),
                 lambda m: gd.periodic_program(m, 3), gd.poisson1d_program):
        import basilisk_b200 as bmg
        bmg.set_tolerance(1e-3)
        oracle.set_globals(1, tolerance=1e-3); oracle.set_globals(2, tolerance=1e-3)
        oracle.set_globals(3, tolerance=1e-3)
        lo, og = prog(omake)
        lg, gg = prog(gpu_make(relax))
        assert lg == lo
        assert np.array_equal(gg.get_a(), og.get_a())
    bmg.set_tolerance(1e-3)


def test_golden_converged_errors_on_gpu():
    """With red-black smoothing the converged errors of the reference's
    programs equal the reference's golden values."""
    import json, os
    import golden_drivers as gd
    import basilisk_b200 as bmg
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")))
    lines, _ = gd.poisson_program(gpu_make("rbgs"), 2)
    assert lines[-1] == gold["poisson_2d"]["lines"][-1]
    lines, _ = gd.variable_program(gpu_make("rbgs"))
    assert lines[-1] == gold["variable_2d"]["lines"][-1]
    lines, _ = gd.periodic_program(gpu_make("rbgs"), 2)
    assert lines == gold["periodic_2d"]["lines"]
    bmg.set_tolerance(1e-3)


# ---- failure paths (host-side, no device fault) -----------------------

def test_nitermax_exhaustion_reports_status():
    import basilisk_b200 as bmg
    rng = np.random.default_rng(12)
    prob = random_problem(2, 6, rng, bc={s: ("dirichlet", 0.0) for s in range(4)})
    g, a, b, alpha, lam = gpu_grid(prob, relax="jacobi")
    bmg.set_niter(nitermax=2)
    try:
        st = g.poisson(a, b, alpha=alpha, tolerance=1e-14)
    finally:
        bmg.set_niter(nitermax=100)
    assert st["i"] == 2 and st["status"] == bmg._lib.ENOTCONV


def test_nan_rhs_reports_status():
    import basilisk_b200 as bmg
    rng = np.random.default_rng(13)
    prob = random_problem(2, 5, rng, bc={s: ("dirichlet", 0.0) for s in range(4)})
    prob["b"][3, 4] = np.nan
    g, a, b, alpha, lam = gpu_grid(prob, relax="rbgs")
    st = g.poisson(a, b, alpha=alpha, tolerance=1e-6, check_status=False)
    assert st["status"] == bmg._lib.ENAN
    assert st["i"] <= 1


def test_foreign_callbacks_rejected():
    import ctypes
    import basilisk_b200 as bmg
    from basilisk_b200 import _lib
    g = bmg.Grid(2, 3)
    a, b = g.scalar(), g.scalar()
    g.select()
    L = _lib.load()
    al = (_lib.bmg_scalar * 1)(a.scalar)
    bl = (_lib.bmg_scalar * 1)(b.scalar)
    m = _lib.MGSolve()
    m.a = ctypes.cast(al, ctypes.POINTER(_lib.bmg_scalar))
    m.b = ctypes.cast(bl, ctypes.POINTER(_lib.bmg_scalar))
    cb = _lib.RELAX_FN(lambda *args: None)
    m.relax = ctypes.cast(cb, ctypes.c_void_p)
    m.residual = ctypes.cast(L.bmg_residual, ctypes.c_void_p)
    p = _lib.Poisson()
    m.data = ctypes.cast(ctypes.pointer(p), ctypes.c_void_p)
    L.mg_solve(m)
    assert L.bmg_last_error() == _lib.EUNSUPPORTED


def test_bad_handles_rejected():
    import basilisk_b200 as bmg
    from basilisk_b200 import _lib
    g = bmg.Grid(2, 3)
    a = g.scalar()
    v = g.face_vector()
    with pytest.raises(bmg.BMGError):
        g.poisson(a, v.components[0])
    with pytest.raises((ValueError, bmg.BMGError)):
        a.set(np.zeros((3, 3, 3)))


def test_mixed_form_error_on_the_headline_workload():
    """The 2048^2 two-phase workload in the mixed and the plain FP64 forms,
    both driven to a maximum residual of 5e-10 (the FP64 form's own floor on
    this problem is about 2e-10: the residual's rounding, with Laplacian terms
    of order |a|/Delta^2 and a density ratio of 1000): the mixed form's
    solution agrees with the FP64 one to 2e-8 relative (max norm; 5.7e-9
    measured); the difference is that of two solutions at that residual, not
    the FP32 arithmetic (at tolerance 1e-6 both differ by 1.7e-5)."""
    import basilisk_b200 as bmg
    from basilisk_b200 import problems
    prob = problems.two_phase_2d(depth=11, seed=1)
    sols = {}
    bmg.set_niter(nitermax=400)
    try:
        for prec in ("fp64", "mixed"):
            g, a, b, alpha, lam = gpu_grid(prob, relax="rbgs", precision=prec)
            st = g.poisson(a, b, alpha=alpha, lambda_=lam, tolerance=5e-10)
            assert st["resa"] <= 5e-10, (prec, st)
            sols[prec] = a.get()
            g.close()
    finally:
        bmg.set_niter(nitermax=100)
    ref = sols["fp64"]
    rel = np.abs(sols["mixed"] - ref).max() / np.abs(ref).max()
    print("mixed vs fp64 at residual 5e-10: %.3g relative" % rel)
    assert rel <= 2e-8
