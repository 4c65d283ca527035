"""Python translations of the reference's Poisson test programs.

Each driver reproduces one Basilisk test program (cited per function) and
returns the lines it prints to stderr, so that they can be compared with the
reference's golden logs (``tests/golden/reference_logs.json``).  A driver is
given a *grid factory*: ``make(dim, depth, origin)`` returning an object with
the interface of ``oracle.oracle.Grid`` (the CPU oracle) or of
``basilisk_b200.Grid`` (the CUDA library), so the same program runs on both.
"""
import math

import numpy as np

PI = 3.14159265358979   # the reference's pi (common.h:48), not M_PI

# The reference evaluates its test functions with the C library's cos/sin;
# Python's math module calls the same libm, numpy's vector kernels may round
# differently in the last bit, which shows in residuals near 1e-10.
_cos = np.frompyfunc(math.cos, 1, 1)
_sin = np.frompyfunc(math.sin, 1, 1)


def cos(x):
    return np.asarray(_cos(x), dtype=np.float64)


def sin(x):
    return np.asarray(_sin(x), dtype=np.float64)


RIGHT, LEFT, TOP, BOTTOM, FRONT, BACK = range(6)
NEUMANN, DIRICHLET, PERIODIC = 0, 1, 2


def dirichlet_all(g, solution):
    """``a[side] = dirichlet(solution(x, y, z))`` on every side: the value at
    the boundary-face centre (cartesian-common.h:15, qcc boundary_staggering)."""
    for side in range(2 * g.dim):
        x, y, z = g.boundary_points(side)
        g.set_bc(side, DIRICHLET, values=solution(x, y, z))


def poisson_program(make, dim=2, depth=None):
    """test/poisson.c: Dirichlet cos(3πx)cos(3πy)cos(3πz) on [-0.5, 0.5]^d,
    13 direct mg_cycle calls (nrelax 4, minlevel 0), residual after each."""
    depth = depth if depth is not None else (9 if dim <= 2 else 6)
    g = make(dim, depth, (-0.5, -0.5, -0.5))

    def solution(x, y, z):
        return cos(3. * PI * x) * cos(3. * PI * y) * cos(3. * PI * z)

    dirichlet_all(g, solution)
    x, y, z = g.centers()
    b = - 9. * dim * PI * PI * cos(3. * PI * x) * cos(3. * PI * y) * cos(3. * PI * z)
    g.set_b(b)
    g.set_a(np.zeros_like(b))
    g.set_alpha_const(1.0)
    g.set_lambda_const(0.0)
    g.residual()
    maxres = []
    for _ in range(13):
        g.mg_cycle(4, 0, depth)
        maxres.append(g.residual())
    lines = ["%d %.2g" % (i, r) for i, r in enumerate(maxres)]
    err = np.max(np.abs(g.get_a() - solution(x, y, z)))
    lines.append("# max error %g" % err)
    return lines, g


def variable_program(make, depth=9):
    """test/variable.c: alpha = x + y + 2 on faces, Dirichlet
    sin(3πx)sin(3πy), 13 direct mg_cycle calls after restriction({c})."""
    dim = 2
    g = make(dim, depth, (-0.5, -0.5, 0.0))

    def solution(x, y, z):
        return sin(3. * PI * x) * sin(3. * PI * y)

    dirichlet_all(g, solution)
    x, y, z = g.centers()
    b = (-18. * PI ** 2 * sin(3. * PI * x) * sin(3. * PI * y) * (x + y + 2.) +
         3. * PI * cos(3. * PI * x) * sin(3. * PI * y) +
         3. * PI * sin(3. * PI * x) * cos(3. * PI * y))
    g.set_b(b)
    g.set_a(np.zeros_like(b))
    comps = []
    for d in range(dim):
        fx, fy, fz = g.face_centers(d)
        comps.append(fx + fy + 2.)
    g.set_alpha(comps)
    g.set_lambda_const(0.0)
    g.restrict_coefficients()
    g.residual()
    maxres = []
    for _ in range(13):
        g.mg_cycle(4, 0, depth)
        maxres.append(g.residual())
    lines = ["%d %.2g" % (i, r) for i, r in enumerate(maxres)]
    err = np.max(np.abs(g.get_a() - solution(x, y, z)))
    lines.append("# max error %g" % err)
    return lines, g


def periodic_program(make, dim=2, sizes=(8, 16, 32, 64)):
    """test/periodic.c: fully periodic Poisson, TOLERANCE 1e-10, poisson(a, b);
    prints the signed maximum of the mean-free error (utils.h statsf)."""
    lines = []
    g = None
    for n in sizes:
        depth = int(round(math.log2(n)))
        g = make(dim, depth, (0.0, 0.0, 0.0))
        for d in range(dim):
            g.set_periodic(d)
        x, y, z = g.centers()
        g.set_a(np.zeros_like(x))
        g.set_b(4. * dim * PI ** 2 * sin(2. * PI * x) * cos(2. * PI * y) * cos(2. * PI * z))
        g.set_alpha_const(1.0)
        g.set_lambda_const(0.0)
        g.set_tolerance_global(1e-10)
        g.poisson()
        e = g.get_a() + sin(2. * PI * x) * cos(2. * PI * y) * cos(2. * PI * z)
        dv = g.delta ** dim
        s_sum = float(np.sum(dv * e))
        volume = dv * e.size
        e = e - s_sum / volume
        lines.append("%d %g" % (n, float(np.max(e))))
    return lines, g


def poisson1d_program(make, depths=(5, 6, 7, 8)):
    """test/poisson1D.c: multigrid1D, Dirichlet sin(3πx), TOLERANCE 1e-4."""
    lines = []
    g = None
    for depth in depths:
        g = make(1, depth, (-0.5, -0.5, 0.0))

        def solution(x, y, z):
            return sin(3. * PI * x)

        dirichlet_all(g, solution)
        x, y, z = g.centers()
        g.set_b(- (3. * PI) ** 2 * sin(3. * PI * x))
        g.set_a(np.zeros_like(x))
        g.set_alpha_const(1.0)
        g.set_lambda_const(0.0)
        g.set_tolerance_global(1e-4)
        g.poisson()
        err = np.max(np.abs(g.get_a() - solution(x, y, z)))
        lines.append("%d %g" % (depth, err))
    return lines, g


# ---------------------------------------------------------------------
# quadtree programs: a *tree factory* ``make(maxdepth, origin)`` returns an
# object with the interface of ``oracle.tree.Tree`` (the CPU oracle) or of
# ``basilisk_b200.TreeGrid`` (the CUDA library).
# ---------------------------------------------------------------------

def dirichlet_tree(t, solution):
    """``a[side] = dirichlet(solution)`` on every side and level: a tree
    applies the condition on every level (tree_boundary_level)."""
    for l in range(t.depth + 1):
        for side in range(4):
            x, y = t.boundary_points(l, side)
            t.set_bc(side, DIRICHLET, level=l, values=solution(x, y, 0.0))


def set_cells(t, which, func):
    """A cell field from its expression, on every level (only leaf values
    are read by the solver; the others are overwritten by restriction and
    prolongation)."""
    for l in range(t.depth + 1):
        x, y = t.centers(l)
        t.set_level(which, l, func(x, y))


def leaf_max_error(t, which, solution):
    err = 0.0
    for l in range(t.depth + 1):
        leaf = (t.flags(l) & 2) != 0
        if leaf.any():
            x, y = t.centers(l)
            e = np.abs(t.get_level(which, l) - solution(x, y, 0.0))[leaf]
            err = max(err, float(e.max()))
    return err


def circle_refinement(depth):
    """``refine (level < depth - 2 || level <= depth*(1. - sqrt(x*x + y*y)))``
    (test/circle.c:70, z = 0 in two dimensions)."""
    def cond(level, x, y):
        return level < depth - 2 or level <= depth * (1. - math.sqrt(x * x + y * y + 0. * 0.))
    return cond


def circle_program(make, depths=(7, 8, 9, 10), niter=15):
    """test/circle.c: Dirichlet cos(3πx)cos(3πy) on a quadtree refined inside
    a circle, 15 direct mg_cycle calls (nrelax 4, minlevel 0)."""
    from oracle.tree import A, B  # field ids are shared with the library
    lines, t = [], None
    for depth in depths:
        t = make(depth, (-0.5, -0.5))
        t.refine(circle_refinement(depth))

        def solution(x, y, z):
            return cos(3. * PI * x) * cos(3. * PI * y) * cos(3. * PI * z)

        dirichlet_tree(t, solution)
        set_cells(t, B, lambda x, y: - 9. * 2 * PI * PI * cos(3. * PI * x) * cos(3. * PI * y) * cos(3. * PI * 0.))
        set_cells(t, A, lambda x, y: np.zeros_like(x))
        t.set_alpha_const(1.0)
        t.set_lambda_const(0.0)
        t.residual()
        maxres = []
        for _ in range(niter):
            t.mg_cycle(4, 0, t.depth)
            maxres.append(t.residual())
        lines += ["residual %d %d %.1g" % (depth, i, r) for i, r in enumerate(maxres)]
        lines.append("max error %d %g" % (depth, leaf_max_error(t, A, solution)))
    return lines, t


def circle_variable_program(make, depths=(7, 8, 9, 10), niter=13):
    """test/circle-variable.c: alpha = x + y + 2 on the faces, Dirichlet
    sin(3πx)sin(3πy), 13 direct mg_cycle calls after restriction({c})."""
    from oracle.tree import A, B, ALPHA_X, ALPHA_Y
    lines, t = [], None
    for depth in depths:
        t = make(depth, (-0.5, -0.5))
        t.refine(circle_refinement(depth))

        def solution(x, y, z):
            return sin(3. * PI * x) * sin(3. * PI * y)

        dirichlet_tree(t, solution)
        set_cells(t, B, lambda x, y: (-18. * PI ** 2 * sin(3. * PI * x) * sin(3. * PI * y) * (x + y + 2.) +
                                      3. * PI * cos(3. * PI * x) * sin(3. * PI * y) +
                                      3. * PI * sin(3. * PI * x) * cos(3. * PI * y)))
        set_cells(t, A, lambda x, y: np.zeros_like(x))
        for l in range(t.depth + 1):
            for d, which in ((0, ALPHA_X), (1, ALPHA_Y)):
                fx, fy = t.face_centers(l, d)
                t.set_level(which, l, fx + fy + 2.)
        t.set_lambda_const(0.0)
        t.restrict_coefficients()
        t.residual()
        maxres = []
        for _ in range(niter):
            t.mg_cycle(4, 0, t.depth)
            maxres.append(t.residual())
        lines += ["residual %d %d %.1g" % (depth, i, r) for i, r in enumerate(maxres)]
        lines.append("max error %d %g" % (depth, leaf_max_error(t, A, solution)))
    return lines, t


def band_refinement(depth, base, width=4.0):
    from basilisk_b200.problems import band_refinement as br
    return br(depth, base, width)


def two_phase_tree(t, seed=1):
    """The two-phase variable-coefficient problem (basilisk_b200.problems,
    two_phase_tree) on an already refined tree: Dirichlet a = 0, lambda = 0."""
    from basilisk_b200.problems import two_phase_tree_levels
    from oracle.tree import A, B, ALPHA_X, ALPHA_Y
    lv = two_phase_tree_levels(t.depth, seed)
    for side in range(4):
        t.set_bc(side, DIRICHLET, 0.0)
    for l, (b, ax, ay) in lv.items():
        t.set_level(B, l, b)
        t.set_level(A, l, np.zeros_like(b))
        t.set_level(ALPHA_X, l, ax)
        t.set_level(ALPHA_Y, l, ay)
    t.set_lambda_const(0.0)
    return t
