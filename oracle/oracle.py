"""ctypes front end of the CPU oracle (``liboracle{1,2,3}d.so``).

TEST INFRASTRUCTURE ONLY.  The oracle is a plain-C restatement of the
reference's multigrid Poisson--Helmholtz solver (Basilisk ``poisson.h`` on
``grid/multigrid.h`` levels); this module lets ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg drive it.
The product package never imports it.

Array conventions follow ``mg_oracle.h``: finest-level arrays without ghosts,
C order with the last index contiguous, face component ``d`` with ``n + 1``
entries along ``d``.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

RIGHT, LEFT, TOP, BOTTOM, FRONT, BACK = range(6)
NEUMANN, DIRICHLET, PERIODIC = 0, 1, 2
RELAX_GS, RELAX_JACOBI, RELAX_RBGS = 0, 1, 2
A, B, RES, LAMBDA, ALPHA_X, ALPHA_Y, ALPHA_Z, DA, UF_X, UF_Y, UF_Z, U_X, U_Y, U_Z, MU_X, MU_Y, MU_Z, RHO = range(18)


class MGStats(ctypes.Structure):
    """Same field order as ``mgstats`` (poisson.h:108-114)."""
    _fields_ = [("i", ctypes.c_int), ("resb", ctypes.c_double),
                ("resa", ctypes.c_double), ("sum", ctypes.c_double),
                ("nrelax", ctypes.c_int), ("minlevel", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_libs = {}


def build():
    """Compile the three oracle libraries (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(dim):
    if dim in _libs:
        return _libs[dim]
    path = os.path.join(HERE, "liboracle%dd.so" % dim)
    if not os.path.exists(path):
        build()
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    D = ctypes.c_double
    I = ctypes.c_int
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "og_new": (P, [I, D, D, D, D]),
        "og_free": (None, [P]),
        "og_set_periodic": (None, [P, I]),
        "og_set_bc": (None, [P, I, I, D, DP]),
        "og_set_relax": (None, [P, I]),
        "og_set_threads": (None, [I]),
        "og_get_threads": (I, []),
        "og_set_field": (None, [P, I, DP]),
        "og_get_field": (None, [P, I, DP]),
        "og_set_alpha_const": (None, [P, D]),
        "og_set_lambda_const": (None, [P, D]),
        "og_restrict_coefficients": (None, [P]),
        "og_residual": (D, [P]),
        "og_mg_cycle": (None, [P, I, I, I]),
        "og_mg_solve": (MGStats, [P, D, I, I]),
        "og_poisson": (MGStats, [P, D, I, I]),
        "og_project": (MGStats, [P, D, I]),
        "og_set_visc_bc": (None, [P, I, I, I, D]),
        "og_set_mu_const": (None, [P, D]),
        "og_set_rho_const": (None, [P, D]),
        "og_viscosity": (MGStats, [P, D, I]),
        "og_residual_viscosity": (D, [P, D]),
        "og_sum_b": (D, [P]),
        "og_get_level": (None, [P, I, I, DP]),
        "og_set_level": (None, [P, I, I, DP]),
        "og_relax_level": (None, [P, I]),
        "og_boundary_level": (None, [P, I, I, I]),
        "og_restrict_res": (None, [P]),
        "og_dimension": (I, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _libs[dim] = L
    return L


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def face_shape(n, dim, d):
    return tuple(n + 1 if e == d else n for e in range(dim))


class Grid:
    """One oracle grid: levels 0..depth of a ``dim``-dimensional box."""

    def __init__(self, dim, depth, L0=1.0, origin=(0.0, 0.0, 0.0),
                 relax=RELAX_GS, threads=1):
        self.dim, self.depth, self.n = dim, depth, 1 << depth
        self.L0, self.origin = L0, tuple(origin) + (0.0,) * (3 - len(origin))
        self.L = lib(dim)
        self.L.og_set_threads(threads)
        self.g = self.L.og_new(depth, L0, *self.origin[:3])
        if not self.g:
            raise ValueError("bad depth %d" % depth)
        self.L.og_set_relax(self.g, relax)
        self._keep = []

    def __del__(self):
        try:
            if self.g:
                self.L.og_free(self.g)
                self.g = None
        except Exception:
            pass

    # ---- geometry helpers (cartesian-common.h:10-34) ----
    @property
    def delta(self):
        return self.L0 * (1.0 / (1 << self.depth))

    def centers(self):
        """Cell-centre coordinates x, y, z (arrays of the cell shape)."""
        n, D = self.n, self.delta
        ax = [(np.arange(n) + 0.5) * D + self.origin[d] for d in range(self.dim)]
        grids = list(np.meshgrid(*ax, indexing="ij"))
        while len(grids) < 3:
            grids.append(np.zeros_like(grids[0]))
        return grids

    def face_centers(self, d):
        """Coordinates of the faces of component d: x = (i/2 + I + .5)Δ - Δ/2 along d."""
        n, D = self.n, self.delta
        ax = []
        for e in range(self.dim):
            if e == d:
                ax.append((np.arange(n + 1) - 0.5 + 0.5) * D + self.origin[e])
            else:
                ax.append((np.arange(n) + 0.5) * D + self.origin[e])
        grids = list(np.meshgrid(*ax, indexing="ij"))
        while len(grids) < 3:
            grids.append(np.zeros_like(grids[0]))
        return grids

    def boundary_points(self, side):
        """Face-centre coordinates of the boundary faces of ``side``
        (x = (ig/2 + I + 0.5)Δ + X0 with ig = ±1, cartesian-common.h:15)."""
        n, D, dim = self.n, self.delta, self.dim
        d, plus = side // 2, side % 2 == 0
        I = n - 1 if plus else 0
        ig = 1 if plus else -1
        coords = []
        tang = [e for e in range(dim) if e != d]
        axes = [(np.arange(n) + 0.5) * D + self.origin[e] for e in tang]
        mesh = np.meshgrid(*axes, indexing="ij") if axes else []
        shape = (n,) * (dim - 1) if dim > 1 else ()
        m = 0
        for e in range(3):
            if e == d:
                coords.append(np.full(shape, (ig / 2.0 + I + 0.5) * D + self.origin[e]))
            elif e < dim:
                coords.append(mesh[m]); m += 1
            else:
                coords.append(np.zeros(shape))
        return coords

    # ---- setup ----
    def set_periodic(self, d):
        self.L.og_set_periodic(self.g, d)

    def set_bc(self, side, kind, value=0.0, values=None):
        if values is not None:
            v = np.ascontiguousarray(values, dtype=np.float64).ravel()
            self._keep.append(v)
            self.L.og_set_bc(self.g, side, kind, value, _ptr(v))
        else:
            self.L.og_set_bc(self.g, side, kind, value, None)

    def set(self, which, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self.L.og_set_field(self.g, which, _ptr(a))

    def get(self, which):
        if which in (ALPHA_X, ALPHA_Y, ALPHA_Z):
            shape = face_shape(self.n, self.dim, which - ALPHA_X)
        elif which in (UF_X, UF_Y, UF_Z):
            shape = face_shape(self.n, self.dim, which - UF_X)
        elif which in (MU_X, MU_Y, MU_Z):
            shape = face_shape(self.n, self.dim, which - MU_X)
        else:
            shape = (self.n,) * self.dim
        out = np.empty(shape, dtype=np.float64)
        self.L.og_get_field(self.g, which, _ptr(out))
        return out

    def get_level(self, which, level):
        n = 1 << level
        if which in (ALPHA_X, ALPHA_Y, ALPHA_Z):
            shape = face_shape(n, self.dim, which - ALPHA_X)
        else:
            shape = (n,) * self.dim
        out = np.empty(shape, dtype=np.float64)
        self.L.og_get_level(self.g, which, level, _ptr(out))
        return out

    def set_level(self, which, level, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self.L.og_set_level(self.g, which, level, _ptr(a))

    def set_a(self, arr):
        self.set(A, arr)

    def set_b(self, arr):
        self.set(B, arr)

    def get_a(self):
        return self.get(A)

    def get_res(self):
        return self.get(RES)

    def set_tolerance_global(self, t):
        set_globals(self.dim, tolerance=t)

    def set_alpha(self, comps):
        for d, c in enumerate(comps):
            self.set(ALPHA_X + d, c)

    def set_alpha_const(self, v):
        self.L.og_set_alpha_const(self.g, v)

    def set_lambda(self, arr):
        self.set(LAMBDA, arr)

    def set_lambda_const(self, v):
        self.L.og_set_lambda_const(self.g, v)

    # ---- solver entry points ----
    def residual(self):
        return self.L.og_residual(self.g)

    def mg_cycle(self, nrelax, minlevel, maxlevel):
        self.L.og_mg_cycle(self.g, nrelax, minlevel, maxlevel)

    def restrict_coefficients(self):
        self.L.og_restrict_coefficients(self.g)

    def mg_solve(self, tolerance=0.0, nrelax=0, minlevel=0):
        return self.L.og_mg_solve(self.g, tolerance, nrelax, minlevel).as_dict()

    def poisson(self, tolerance=0.0, nrelax=0, minlevel=0):
        return self.L.og_poisson(self.g, tolerance, nrelax, minlevel).as_dict()

    def set_uf(self, comps):
        for d, c in enumerate(comps):
            self.set(UF_X + d, c)

    def get_uf(self):
        return [self.get(UF_X + d) for d in range(self.dim)]

    def set_u(self, comps):
        for d, c in enumerate(comps):
            self.set(U_X + d, c)

    def get_u(self):
        return [self.get(U_X + d) for d in range(self.dim)]

    def set_mu(self, comps):
        for d, c in enumerate(comps):
            self.set(MU_X + d, c)

    def set_mu_const(self, v):
        self.L.og_set_mu_const(self.g, float(v))

    def set_rho(self, arr):
        self.set(RHO, arr)

    def set_rho_const(self, v):
        self.L.og_set_rho_const(self.g, float(v))

    def set_visc_bc(self, comp, side, kind, value=0.0):
        self.L.og_set_visc_bc(self.g, comp, side, kind, float(value))

    def viscosity(self, dt, nrelax=0):
        """viscosity (u, mu, rho, dt, nrelax) (viscosity.h:169-183)."""
        return self.L.og_viscosity(self.g, dt, nrelax).as_dict()

    def residual_viscosity(self, dt):
        return self.L.og_residual_viscosity(self.g, dt)

    def project(self, dt=0.0, nrelax=0):
        """project (uf, p = a, alpha, dt, nrelax) (poisson.h:468-509)."""
        return self.L.og_project(self.g, dt, nrelax).as_dict()

    def sum_b(self):
        return self.L.og_sum_b(self.g)


def set_globals(dim, tolerance=None, nitermax=None, nitermin=None):
    L = lib(dim)
    if tolerance is not None:
        ctypes.c_double.in_dll(L, "og_TOLERANCE").value = tolerance
    if nitermax is not None:
        ctypes.c_int.in_dll(L, "og_NITERMAX").value = nitermax
    if nitermin is not None:
        ctypes.c_int.in_dll(L, "og_NITERMIN").value = nitermin


def get_tolerance(dim):
    return ctypes.c_double.in_dll(lib(dim), "og_TOLERANCE").value
