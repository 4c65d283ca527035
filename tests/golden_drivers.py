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
