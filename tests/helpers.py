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
