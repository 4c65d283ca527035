"""viscosity () (viscosity.h:169-183): the oracle's smoothers reach the same
discrete solution, and the CUDA path gives the oracle's result bit for bit
(FP64, same smoother).  The reference's own tests of viscosity () are full
physics programs (test/axi.c, fall.c, gaussian.c) outside this path, so
the operator (viscosity.h:25-160, restated in the oracle) is pinned by a
closed-form known answer: on a periodic box a sum of Fourier modes is
mapped by the discrete operator to M U cos(phi) with M the operator's
symbol, so both the oracle and the CUDA path must return the mode sum from
its image (fourier_case)."""
import numpy as np
import pytest

from oracle import oracle


def shape(n, dim, d=None):
    return tuple(n + 1 if e == d else n for e in range(dim))


def oracle_visc(dim, depth, relax, periodic, mu, rho, seed, dt=1e-2):
    n = 1 << depth
    rng = np.random.default_rng(seed)
    g = oracle.Grid(dim, depth, relax=relax)
    u = [rng.standard_normal(shape(n, dim)) for _ in range(dim)]
    if periodic:
        for d in range(dim):
            g.set_periodic(d)
    else:
        for c in range(dim):
            for side in range(2 * dim):
                # no slip on the walls: Dirichlet 0 for every component
                g.set_visc_bc(c, side, oracle.DIRICHLET, 0.0)
    g.set_u(u)
    m = None
    if mu == "field":
        m = [rng.uniform(0.5, 1.5, shape(n, dim, d)) for d in range(dim)]
        if periodic:
            for d in range(dim):
                sn = [slice(None)] * dim
                s0 = [slice(None)] * dim
                sn[d], s0[d] = n, 0
                m[d][tuple(sn)] = m[d][tuple(s0)]
        g.set_mu(m)
    else:
        g.set_mu_const(0.7)
    r = None
    if rho == "field":
        r = rng.uniform(0.5, 2.0, shape(n, dim))
        g.set_rho(r)
    else:
        g.set_rho_const(1.3)
    return g, u, m, r


def fourier_case(dim, depth, seed, mu=0.7, rho=1.3, dt=1e-2, modes=4):
    """A known answer independent of any stencil code.  With constant mu and
    rho on a periodic grid, the discrete operator of residual_viscosity
    (viscosity.h:127-146, lambda = 1),

        (A u)_c = u_c - dt/(rho Delta^2) B_c(u),

    maps the mode u_e = U_e cos(phi), phi = sum_d theta_d i_d + psi, theta_d =
    2 pi k_d / n, to (A u)_c = M_ce U_e cos(phi) with the symmetric matrix

        M_cc = 1 + C (8 s_c^2 + 4 sum_{d != c} s_d^2),   s_d = sin(theta_d/2)
        M_ce = C sin(theta_c) sin(theta_e)              (c != e)

    C = dt mu/(rho Delta^2): the second differences along c (weight 2 mu) and
    across (weight mu) give the diagonal, and the four-point cross terms
    (u_e[1,1] - u_e[-1,1] - u_e[1,-1] + u_e[-1,-1])/4 the off-diagonal.
    Returns (u_exact, A u_exact) as lists of dim arrays."""
    n = 1 << depth
    rng = np.random.default_rng(seed)
    C = dt * mu / (rho * (1.0 / n) ** 2)
    idx = np.meshgrid(*[np.arange(n)] * dim, indexing="ij")
    u = [np.zeros((n,) * dim) for _ in range(dim)]
    Au = [np.zeros((n,) * dim) for _ in range(dim)]
    for _ in range(modes):
        k = rng.integers(-n // 2 + 1, n // 2, size=dim)
        theta = 2 * np.pi * k / n
        psi = rng.uniform(0, 2 * np.pi)
        U = rng.standard_normal(dim)
        s2 = np.sin(theta / 2) ** 2
        M = np.empty((dim, dim))
        for c in range(dim):
            for e in range(dim):
                M[c, e] = (1 + C * (8 * s2[c] + 4 * (s2.sum() - s2[c]))) if c == e \
                    else C * np.sin(theta[c]) * np.sin(theta[e])
        phi = sum(theta[d] * idx[d] for d in range(dim)) + psi
        cos = np.cos(phi)
        MU = M @ U
        for c in range(dim):
            u[c] += U[c] * cos
            Au[c] += MU[c] * cos
    return u, Au, dict(mu=mu, rho=rho, dt=dt)


@pytest.mark.parametrize("dim,depth", [(2, 4), (2, 6), (3, 3)])
def test_oracle_viscosity_fourier_known_answer(dim, depth):
    """The oracle's residual_viscosity of the exact mode sum is zero to
    round-off, and viscosity () started from u = A u_exact (it solves A u =
    r with r = the input u) returns u_exact: the operator and the solver are
    pinned by the closed-form symbol, not by another restatement."""
    u, Au, p = fourier_case(dim, depth, seed=11 + dim + depth)
    scale = max(np.abs(x).max() for x in Au)
    for relax in (oracle.RELAX_GS, oracle.RELAX_JACOBI, oracle.RELAX_RBGS):
        g = oracle.Grid(dim, depth, relax=relax)
        for d in range(dim):
            g.set_periodic(d)
        g.set_mu_const(p["mu"])
        g.set_rho_const(p["rho"])
        # residual of u_exact with r = A u_exact: viscosity () copies u into r,
        # so set u = A u_exact, let one solve build r, then evaluate at u_exact
        g.set_u(Au)
        old = oracle.get_tolerance(dim)
        oracle.set_globals(dim, tolerance=1e-12)
        try:
            st = g.viscosity(dt=p["dt"])
        finally:
            oracle.set_globals(dim, tolerance=old)
        assert st["resa"] <= 1e-12, st
        sol = g.get_u()
        err = max(np.abs(s - e).max() for s, e in zip(sol, u)) / max(np.abs(e).max() for e in u)
        assert err < 1e-11, (relax, err)
        g.set_u(u)
        res = g.residual_viscosity(p["dt"])
        assert res <= 1e-13 * scale * (1 << depth), res


@pytest.mark.gpu
@pytest.mark.parametrize("dim,depth,relax", [(2, 7, "rbgs"), (3, 4, "jacobi")])
def test_viscosity_gpu_fourier_known_answer(dim, depth, relax):
    """The CUDA path on the same closed-form case: the solve of A u = A
    u_exact returns u_exact."""
    import basilisk_b200 as bmg
    u, Au, p = fourier_case(dim, depth, seed=5 + dim + depth)
    g = bmg.Grid(dim, depth, relax=relax)
    for d in range(dim):
        g.periodic(2 * d)
    uu = g.vector(Au)
    bmg.set_tolerance(1e-12)
    try:
        st = g.viscosity(uu, g.const_face_vector(p["mu"]), g.const_scalar(p["rho"]), p["dt"])
    finally:
        bmg.set_tolerance(1e-3)
    assert st["resa"] <= 1e-12, st
    err = max(np.abs(c.get() - e).max() for c, e in zip(uu, u)) / max(np.abs(e).max() for e in u)
    assert err < 1e-11, err
    g.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_smoothers_reach_the_same_solution(dim):
    depth = 4
    sols = {}
    for relax in (oracle.RELAX_GS, oracle.RELAX_JACOBI, oracle.RELAX_RBGS):
        g, u, m, r = oracle_visc(dim, depth, relax, False, "field", "field", seed=1)
        old = oracle.get_tolerance(dim)
        oracle.set_globals(dim, tolerance=1e-11)
        try:
            st = g.viscosity(dt=1e-2)
        finally:
            oracle.set_globals(dim, tolerance=old)
        assert st["resa"] <= 1e-11, st
        sols[relax] = np.stack(g.get_u())
    ref = sols[oracle.RELAX_GS]
    for relax in (oracle.RELAX_JACOBI, oracle.RELAX_RBGS):
        assert np.abs(sols[relax] - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dim,depth,periodic,mu,rho,relax",
                         [(2, 6, False, "field", "field", "jacobi"),
                          (2, 6, True, "const", "field", "rbgs"),
                          (2, 7, False, "field", "const", "rbgs"),
                          (3, 4, False, "field", "field", "rbgs"),
                          (3, 4, True, "field", "const", "jacobi")])
def test_viscosity_gpu_matches_oracle(dim, depth, periodic, mu, rho, relax):
    import basilisk_b200 as bmg
    orelax = oracle.RELAX_JACOBI if relax == "jacobi" else oracle.RELAX_RBGS
    o, u, m, r = oracle_visc(dim, depth, orelax, periodic, mu, rho, seed=depth + dim)
    g = bmg.Grid(dim, depth, relax=relax)
    if periodic:
        for d in range(dim):
            g.periodic(2 * d)
    uu = g.vector(u)
    if not periodic:
        for c in uu:
            for side in range(2 * dim):
                c.bc(side, "dirichlet", 0.0)
        for c, comp in zip(uu, u):       # ghosts from the new BCs
            c.set(comp)
    mf = g.face_vector(m) if mu == "field" else g.const_face_vector(0.7)
    rf = g.scalar(r) if rho == "field" else g.const_scalar(1.3)
    old = oracle.get_tolerance(dim)
    oracle.set_globals(dim, tolerance=1e-9)
    bmg.set_tolerance(1e-9)
    try:
        so = o.viscosity(dt=1e-2)
        sg = g.viscosity(uu, mf, rf, 1e-2)
    finally:
        oracle.set_globals(dim, tolerance=old)
        bmg.set_tolerance(1e-3)
    for k in ("i", "nrelax", "minlevel"):
        assert sg[k] == so[k], (k, sg, so)
    assert sg["resb"] == so["resb"] and sg["resa"] == so["resa"], (sg, so)
    assert abs(sg["sum"] - so["sum"]) <= 1e-12 * max(1.0, np.abs(np.stack(u)).sum())
    for c, oc in zip(uu, o.get_u()):
        np.testing.assert_array_equal(c.get(), oc)
    g.close()
