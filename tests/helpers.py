"""Shared set-up of one problem on the CPU oracle and on the CUDA library.

A problem is a dict as built by ``basilisk_b200.problems``: dim, depth,
periodic dims, b, alpha (face components or None), lambda (None, a number or
a cell array), bc {side: (kind, value or per-face array)}.
"""
import numpy as np

from oracle import oracle

KIND = {"dirichlet": oracle.DIRICHLET, "neumann": oracle.NEUMANN}


def oracle_grid(prob, relax=oracle.RELAX_JACOBI, threads=1, L0=1.0, origin=(0.0, 0.0, 0.0)):
    g = oracle.Grid(prob["dim"], prob["depth"], L0=L0, origin=origin, relax=relax,
                    threads=threads)
    for d in prob["periodic"]:
        g.set_periodic(d)
    for side, (kind, val) in prob["bc"].items():
        if np.isscalar(val):
            g.set_bc(side, KIND[kind], value=float(val))
        else:
            g.set_bc(side, KIND[kind], values=val)
    g.set_b(prob["b"])
    g.set_a(prob.get("a0", np.zeros(prob["b"].shape)))
    if prob["alpha"] is None:
        g.set_alpha_const(1.0)
    elif np.isscalar(prob["alpha"]):
        g.set_alpha_const(float(prob["alpha"]))
    else:
        g.set_alpha(prob["alpha"])
    lam = prob["lambda"]
    if lam is None:
        g.set_lambda_const(0.0)
    elif np.isscalar(lam):
        g.set_lambda_const(float(lam))
    else:
        g.set_lambda(lam)
    return g


def gpu_grid(prob, relax="jacobi", precision="fp64", graphs=True, L0=1.0,
             origin=(0.0, 0.0, 0.0)):
    import basilisk_b200 as bmg
    g = bmg.Grid(prob["dim"], prob["depth"], L0=L0, origin=origin, relax=relax,
                 precision=precision, graphs=graphs)
    for d in prob["periodic"]:
        g.periodic(2 * d)
    a = g.scalar()
    for side, (kind, val) in prob["bc"].items():
        if np.isscalar(val):
            a.bc(side, kind, float(val))
        else:
            a.bc(side, kind, 0.0, values=val)
    a.set(prob.get("a0", np.zeros(prob["b"].shape)))
    b = g.scalar(prob["b"])
    if prob["alpha"] is None:
        alpha = None
    elif np.isscalar(prob["alpha"]):
        alpha = g.const_face_vector(float(prob["alpha"]))
    else:
        alpha = g.face_vector(prob["alpha"])
    lam = prob["lambda"]
    if lam is None:
        lam_f = None
    elif np.isscalar(lam):
        lam_f = g.const_scalar(float(lam))
    else:
        lam_f = g.scalar(lam)
    return g, a, b, alpha, lam_f


def random_problem(dim, depth, rng, periodic=(), bc=None, alpha="field", lam=None,
                   a0=False):
    """A random well-posed problem for parity tests."""
    n = 1 << depth
    shape = (n,) * dim
    b = rng.standard_normal(shape)
    if alpha == "field":
        al = [rng.uniform(0.5, 2.0, size=tuple(n + 1 if e == d else n for e in range(dim)))
              for d in range(dim)]
    else:
        al = alpha
    if lam == "field":
        lm = -rng.uniform(0.5, 2.0, size=shape)
    else:
        lm = lam
    if bc is None:
        bc = {}
    if len(periodic) == dim and (lm is None or (np.isscalar(lm) and lm == 0)):
        b = b - b.mean()
    prob = {"dim": dim, "depth": depth, "periodic": tuple(periodic), "b": b, "alpha": al,
            "lambda": lm, "bc": bc}
    if a0:
        prob["a0"] = rng.standard_normal(shape)
    return prob


class GpuTree:
    """The interface of ``oracle.tree.Tree`` on the CUDA library's
    ``TreeGrid``, so that the tree programs of ``golden_drivers`` run on
    both; the field ids are the oracle's."""

    def __init__(self, maxdepth, origin=(0.0, 0.0), relax="rbgs", L0=1.0, graphs=True,
                 precision="fp64"):
        import basilisk_b200 as bmg
        from oracle import tree as ot
        self.ot = ot
        self.g = bmg.TreeGrid(maxdepth, L0=L0, origin=origin, relax=relax, graphs=graphs,
                              precision=precision)
        self.L0, self.X0, self.Y0 = float(L0), float(origin[0]), float(origin[1])
        self.f = {ot.A: self.g.scalar(), ot.B: self.g.scalar(), ot.RES: self.g.scalar(),
                  ot.DA: self.g.scalar()}
        self.alpha = None
        self.lam = None

    def close(self):
        self.g.close()

    def refine(self, cond):
        return self.g.refine(cond)

    @property
    def depth(self):
        return self.g.tree_depth

    @property
    def leaves(self):
        return self.g.leaves

    def flags(self, level):
        return self.g.flags(level)

    def delta(self, level):
        return self.L0 * (1.0 / (1 << level))

    # geometry shared with the oracle's Tree
    def centers(self, level):
        return self.ot.Tree.centers(self, level)

    def face_centers(self, level, d):
        return self.ot.Tree.face_centers(self, level, d)

    def boundary_points(self, level, side):
        return self.ot.Tree.boundary_points(self, level, side)

    def _field(self, which):
        ot = self.ot
        if which == ot.LAMBDA:
            if self.lam is None or self.lam.const is not None:
                self.lam = self.g.scalar()
            return self.lam
        if which in (ot.ALPHA_X, ot.ALPHA_Y):
            if self.alpha is None or self.alpha.const is not None:
                self.alpha = self.g.face_vector()
            return self.alpha.components[0 if which == ot.ALPHA_X else 1]
        return self.f[which]

    def set_level(self, which, level, values):
        self._field(which).set(np.ascontiguousarray(values, dtype=np.float64), level=level)

    def get_level(self, which, level):
        return self._field(which).get(level=level)

    def set_bc(self, side, kind, value=0.0, level=None, values=None):
        ot = self.ot
        k = "dirichlet" if kind == ot.DIRICHLET else "neumann"
        if values is None:
            self.f[ot.A].bc(side, k, float(value))
        else:
            self.f[ot.A].bc_level(side, k, level, values)
        self.f[ot.DA].bc(side, k, 0.0)

    def set_relax(self, mode):
        ot = self.ot
        self.g.set_relax({ot.RELAX_RBGS: "rbgs", ot.RELAX_JACOBI: "jacobi"}[mode])

    def set_alpha_const(self, v):
        self.alpha = None if v == 1.0 else self.g.const_face_vector(v)

    def set_lambda_const(self, v):
        self.lam = None if v == 0.0 else self.g.const_scalar(v)

    def restrict_coefficients(self):
        fs = [f for f in (self.alpha, self.lam) if f is not None and f.const is None]
        if fs:
            self.g.restriction(fs)

    def residual(self):
        ot = self.ot
        return self.g.residual(self.f[ot.A], self.f[ot.B], self.f[ot.RES], self.alpha, self.lam)

    def mg_cycle(self, nrelax, minlevel, maxlevel):
        ot = self.ot
        self.g.mg_cycle(self.f[ot.A], self.f[ot.RES], self.f[ot.DA], nrelax, minlevel, maxlevel,
                        self.alpha, self.lam)

    def mg_solve(self, tolerance=0.0, nrelax=4, minlevel=0):
        ot = self.ot
        return self.g.mg_solve(self.f[ot.A], self.f[ot.B], self.alpha, self.lam,
                               tolerance=tolerance, nrelax=nrelax, minlevel=minlevel)

    def poisson(self, tolerance=0.0, nrelax=4, minlevel=0):
        ot = self.ot
        return self.g.poisson(self.f[ot.A], self.f[ot.B], self.alpha, self.lam,
                              tolerance=tolerance, nrelax=nrelax, minlevel=minlevel)
