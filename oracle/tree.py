"""ctypes front end of the quadtree CPU oracle (``liboracletree.so``).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's tree
multigrid (Basilisk ``poisson.h`` on ``grid/quadtree.h``) in plain C; this
module lets ``tests/`` and ``bench.py``'s CPU-baseline leg drive it.  The
product package never imports it.

Level arrays are the interior ``n x n`` values of one level (C order, the y
index contiguous); x faces are ``(n+1) x n``, y faces ``n x (n+1)``.
"""
import ctypes
import os

import numpy as np

from . import oracle as _og

HERE = os.path.dirname(os.path.abspath(__file__))

ACTIVE, LEAF, HALO, PROL = 1, 2, 4, 8
RIGHT, LEFT, TOP, BOTTOM = range(4)
NEUMANN, DIRICHLET = 0, 1
RELAX_GS, RELAX_JACOBI, RELAX_RBGS = 0, 1, 2
A, B, RES, LAMBDA, ALPHA_X, ALPHA_Y, DA = range(7)

COND = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                        ctypes.c_void_p)

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "liboracletree.so")
    if not os.path.exists(path):
        _og.build()
    L = ctypes.CDLL(path)
    P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    DP = ctypes.POINTER(ctypes.c_double)
    UP = ctypes.POINTER(ctypes.c_ubyte)
    sig = {
        "ot_new": (P, [I, D, D, D]),
        "ot_free": (None, [P]),
        "ot_refine": (I, [P, COND, P]),
        "ot_depth": (I, [P]),
        "ot_leaves": (ctypes.c_long, [P]),
        "ot_get_flags": (None, [P, I, UP]),
        "ot_set_relax": (None, [P, I]),
        "ot_set_bc": (None, [P, I, I, D, I, DP]),
        "ot_set_level": (None, [P, I, I, DP]),
        "ot_get_level": (None, [P, I, I, DP]),
        "ot_set_alpha_const": (None, [P, D]),
        "ot_set_lambda_const": (None, [P, D]),
        "ot_restrict_coefficients": (None, [P]),
        "ot_boundary": (None, [P, I, I, I]),
        "ot_relax_level": (None, [P, I]),
        "ot_residual": (D, [P]),
        "ot_sum_b": (D, [P]),
        "ot_mg_cycle": (None, [P, I, I, I]),
        "ot_mg_solve": (_og.MGStats, [P, D, I, I]),
        "ot_poisson": (_og.MGStats, [P, D, I, I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def set_niter(nitermax=None, nitermin=None):
    """The tree oracle's NITERMAX / NITERMIN (poisson.h:102)."""
    L = lib()
    if nitermax is not None:
        ctypes.c_int.in_dll(L, "ot_NITERMAX").value = nitermax
    if nitermin is not None:
        ctypes.c_int.in_dll(L, "ot_NITERMIN").value = nitermin


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Tree:
    """A quadtree on the oracle: ``init_grid (1)`` then ``refine (cond)``."""

    def __init__(self, maxdepth, L0=1.0, origin=(0.0, 0.0)):
        self.L = lib()
        self.maxdepth = maxdepth
        self.L0 = float(L0)
        self.X0, self.Y0 = float(origin[0]), float(origin[1])
        self.h = self.L.ot_new(maxdepth, self.L0, self.X0, self.Y0)
        if not self.h:
            raise ValueError("bad maxdepth %d" % maxdepth)

    def close(self):
        if self.h:
            self.L.ot_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # -- mesh ---------------------------------------------------------
    def refine(self, cond):
        """``cond(level, x, y) -> bool`` evaluated on leaves until no leaf
        asks for refinement (tree-common.h:308-326)."""
        cb = COND(lambda l, x, y, d: 1 if cond(l, x, y) else 0)
        r = self.L.ot_refine(self.h, cb, None)
        if r < 0:
            raise ValueError("refinement past maxdepth %d" % self.maxdepth)
        return r

    @property
    def depth(self):
        return self.L.ot_depth(self.h)

    @property
    def leaves(self):
        return self.L.ot_leaves(self.h)

    def flags(self, level):
        n = 1 << level
        out = np.zeros((n, n), dtype=np.uint8)
        self.L.ot_get_flags(self.h, level, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
        return out

    def delta(self, level):
        return self.L0 * (1.0 / (1 << level))

    def centers(self, level):
        n = 1 << level
        D = self.delta(level)
        c = (np.arange(n) + 0.5) * D
        x, y = np.meshgrid(c + self.X0, c + self.Y0, indexing="ij")
        return x, y

    def face_centers(self, level, d):
        n = 1 << level
        D = self.delta(level)
        if d == 0:
            xi = np.arange(n + 1) * D + self.X0
            yj = (np.arange(n) + 0.5) * D + self.Y0
        else:
            xi = (np.arange(n) + 0.5) * D + self.X0
            yj = np.arange(n + 1) * D + self.Y0
        x, y = np.meshgrid(xi, yj, indexing="ij")
        return x, y

    def boundary_points(self, level, side):
        """Centres of the boundary faces of one level, over the tangential
        index (where dirichlet () evaluates its expression)."""
        n = 1 << level
        D = self.delta(level)
        t = (np.arange(n) + 0.5) * D
        if side == RIGHT:
            return np.full(n, self.X0 + n * D), t + self.Y0
        if side == LEFT:
            return np.full(n, self.X0), t + self.Y0
        if side == TOP:
            return t + self.X0, np.full(n, self.Y0 + n * D)
        return t + self.X0, np.full(n, self.Y0)

    # -- fields -------------------------------------------------------
    def set_level(self, which, level, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.L.ot_set_level(self.h, which, level, _dp(v))

    def get_level(self, which, level):
        n = 1 << level
        shape = (n + 1, n) if which == ALPHA_X else (n, n + 1) if which == ALPHA_Y else (n, n)
        out = np.zeros(shape)
        self.L.ot_get_level(self.h, which, level, _dp(out))
        return out

    def set_bc(self, side, kind, value=0.0, level=None, values=None):
        if values is None:
            self.L.ot_set_bc(self.h, side, kind, float(value), 0, None)
        else:
            v = np.ascontiguousarray(values, dtype=np.float64)
            self.L.ot_set_bc(self.h, side, kind, 0.0, level, _dp(v))

    def set_relax(self, mode):
        self.L.ot_set_relax(self.h, mode)

    def set_alpha_const(self, v):
        self.L.ot_set_alpha_const(self.h, float(v))

    def set_lambda_const(self, v):
        self.L.ot_set_lambda_const(self.h, float(v))

    def restrict_coefficients(self):
        self.L.ot_restrict_coefficients(self.h)

    def residual(self):
        return self.L.ot_residual(self.h)

    def mg_cycle(self, nrelax, minlevel, maxlevel):
        self.L.ot_mg_cycle(self.h, nrelax, minlevel, maxlevel)

    def mg_solve(self, tolerance=0.0, nrelax=4, minlevel=0):
        return self.L.ot_mg_solve(self.h, tolerance, nrelax, minlevel).as_dict()

    def poisson(self, tolerance=0.0, nrelax=4, minlevel=0):
        return self.L.ot_poisson(self.h, tolerance, nrelax, minlevel).as_dict()

    def leaf_values(self, which):
        """(level, values) pairs of a cell field on the leaves of each level."""
        out = []
        for l in range(self.depth + 1):
            f = self.flags(l)
            m = (f & LEAF) != 0
            if m.any():
                out.append((l, self.get_level(which, l)[m]))
        return out
