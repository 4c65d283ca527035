"""project () (poisson.h:468-509): the reference's test/solenoidal.c line on
the oracle, the discrete divergence after projection, and the CUDA path bit
for bit against the oracle."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
PI = 3.14159265358979   # common.h:48


def taylor_green(g):
    """test/solenoidal.c: uf.x = -cos(2 pi x) sin(2 pi y), uf.y = sin(2 pi x)
    cos(2 pi y) at the face centres (libm cos/sin)."""
    comps = []
    for d, f in ((0, lambda x, y: -math.cos(2. * PI * x) * math.sin(2. * PI * y)),
                 (1, lambda x, y: math.sin(2. * PI * x) * math.cos(2. * PI * y))):
        fx, fy, _ = g.face_centers(d)
        comps.append(np.vectorize(f)(fx, fy))
    return comps


def divergence(u):
    dim = len(u)
    out = None
    for e in range(dim):
        sl_hi = [slice(None)] * dim
        sl_lo = [slice(None)] * dim
        sl_hi[e] = slice(1, None)
        sl_lo[e] = slice(None, -1)
        term = u[e][tuple(sl_hi)] - u[e][tuple(sl_lo)]
        out = term if out is None else out + term
    return out


def test_solenoidal_log_line():
    """test/solenoidal.c (2D): init_grid (8), periodic, TOLERANCE = 1e-10,
    project (uf, p): 'div max before: 0.000000000' (test/solenoidal.ref)."""
    g = oracle.Grid(2, 3, origin=(-0.5, -0.5))
    g.set_periodic(0)
    g.set_periodic(1)
    g.set_uf(taylor_green(g))
    g.set_a(np.zeros((8, 8)))
    g.set_alpha_const(1.0)
    g.set_lambda_const(0.0)
    old = oracle.get_tolerance(2)
    oracle.set_globals(2, tolerance=1e-10)
    try:
        g.project()
    finally:
        oracle.set_globals(2, tolerance=old)
    line = "div max before: %.9f" % np.abs(divergence(g.get_uf())).max()
    ref = json.load(open(os.path.join(HERE, "golden", "reference_logs.json")))
    assert line == ref["solenoidal_2d"]["lines"][0]


@pytest.mark.parametrize("periodic", [True, False])
def test_projection_removes_divergence(periodic):
    """A random face field: after project (dt = 0.5) the discrete divergence
    is at the tolerance's level (|div| dt <= TOLERANCE up to the residual's
    1/Delta^2 scale)."""
    rng = np.random.default_rng(7)
    depth, n = 5, 32
    g = oracle.Grid(2, depth, relax=oracle.RELAX_RBGS)
    if periodic:
        g.set_periodic(0)
        g.set_periodic(1)
    else:
        for side in range(4):
            g.set_bc(side, oracle.NEUMANN, value=0.0)
    u = [rng.standard_normal((n + 1, n)), rng.standard_normal((n, n + 1))]
    if periodic:
        u[0][n] = u[0][0]
        u[1][:, n] = u[1][:, 0]
    else:
        u[0][0] = u[0][n] = 0.0      # no flow through the walls
        u[1][:, 0] = u[1][:, n] = 0.0
    g.set_uf(u)
    g.set_a(np.zeros((n, n)))
    g.set_alpha_const(1.0)
    g.set_lambda_const(0.0)
    old = oracle.get_tolerance(2)
    oracle.set_globals(2, tolerance=1e-9)
    try:
        st = g.project(dt=0.5)
    finally:
        oracle.set_globals(2, tolerance=old)
    div = divergence(g.get_uf()) / (0.5 * g.delta)
    before = np.abs(divergence(u)).max() / (0.5 * g.delta)
    assert st["resa"] <= 1e-9 / 0.25
    assert np.abs(div).max() <= 1e-9 / 0.25 * 1.001 and before > 1.0


def gpu_project(dim, depth, periodic, dt, alpha, relax, seed):
    import basilisk_b200 as bmg
    rng = np.random.default_rng(seed)
    n = 1 << depth
    g = bmg.Grid(dim, depth, relax=relax)
    o = oracle.Grid(dim, depth, relax=oracle.RELAX_JACOBI if relax == "jacobi" else oracle.RELAX_RBGS)
    if periodic:
        for d in range(dim):
            g.periodic(2 * d)
            o.set_periodic(d)
    p = g.scalar()
    if not periodic:
        for side in range(2 * dim):
            p.bc(side, "dirichlet", 0.0)
            o.set_bc(side, oracle.DIRICHLET, value=0.0)
    shape = lambda d: tuple(n + 1 if e == d else n for e in range(dim))
    u = [rng.standard_normal(shape(d)) for d in range(dim)]
    if periodic:
        for d in range(dim):
            sl_n = [slice(None)] * dim
            sl_0 = [slice(None)] * dim
            sl_n[d], sl_0[d] = n, 0
            u[d][tuple(sl_n)] = u[d][tuple(sl_0)]
    uf = g.face_vector(u)
    o.set_uf(u)
    o.set_a(np.zeros((n,) * dim))
    o.set_lambda_const(0.0)
    al = None
    if alpha == "field":
        a = [rng.uniform(0.5, 2.0, size=shape(d)) for d in range(dim)]
        if periodic:
            for d in range(dim):
                sl_n = [slice(None)] * dim
                sl_0 = [slice(None)] * dim
                sl_n[d], sl_0[d] = n, 0
                a[d][tuple(sl_n)] = a[d][tuple(sl_0)]
        al = g.face_vector(a)
        o.set_alpha(a)
    else:
        o.set_alpha_const(1.0)
    sg = g.project(uf, p, alpha=al, dt=dt)
    so = o.project(dt=dt)
    return g, uf, p, o, sg, so


@pytest.mark.gpu
@pytest.mark.parametrize("dim,depth,periodic,alpha,relax",
                         [(2, 6, True, None, "jacobi"), (2, 6, False, "field", "rbgs"),
                          (3, 4, True, "field", "rbgs"), (2, 7, False, None, "jacobi")])
def test_project_gpu_matches_oracle(dim, depth, periodic, alpha, relax):
    """The CUDA project () gives the oracle's pressure, corrected faces and
    statistics bit for bit (FP64, same smoother)."""
    g, uf, p, o, sg, so = gpu_project(dim, depth, periodic, 0.25, alpha, relax, seed=depth)
    for k in ("i", "nrelax", "minlevel"):
        assert sg[k] == so[k], k
    assert sg["resb"] == so["resb"] and sg["resa"] == so["resa"]
    np.testing.assert_array_equal(p.get(), o.get_a())
    for d, c in enumerate(uf.get()):
        np.testing.assert_array_equal(c, o.get_uf()[d])
    g.close()
