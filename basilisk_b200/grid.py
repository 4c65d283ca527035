"""Python front end of the B200 multigrid Poisson--Helmholtz solver.

It mirrors the reference's Python binding of this path (Basilisk
``poisson.i``: ``poisson(a, b, alpha=None, lambda0=0, tolerance=1e-3)``
returning ``mgstats``) over the C-ABI of ``libbmg.so``: a ``Grid`` plays the
role of Basilisk's global grid (``init_grid``), ``Scalar`` / ``FaceVector``
the role of ``scalar`` / ``face vector`` fields.  Every computation runs in
the library's CUDA kernels; this module only moves arrays in and out.

Arrays are finest-level values without ghosts, in C order with the last index
contiguous (the reference's index order); face component ``d`` has ``n + 1``
entries along ``d``.  numpy arrays go through host memory, CUDA torch tensors
are read and written in place on the device.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import check, bmg_scalar, bmg_vector

SIDES = {"right": 0, "left": 1, "top": 2, "bottom": 3, "front": 4, "back": 5}
KINDS = {"neumann": _lib.NEUMANN, "dirichlet": _lib.DIRICHLET}


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _side(s):
    return SIDES[s] if isinstance(s, str) else int(s)


class Field:
    def __init__(self, grid, handle, face_dim=-1, const=None):
        self.grid, self.handle, self.face_dim, self.const = grid, handle, face_dim, const

    @property
    def scalar(self):
        return bmg_scalar(self.handle)

    def shape(self, level=None):
        n = 1 << (self.grid.depth if level is None else level)
        return tuple(n + 1 if e == self.face_dim else n for e in range(self.grid.dim))

    def set(self, values, level=None):
        """Set the values of the finest level (or of ``level``)."""
        g = self.grid
        lvl = g.depth if level is None else level
        shape = self.shape(lvl)
        L = _lib.load()
        if _is_torch(values) and values.is_cuda:
            import torch
            v = values.detach().to(torch.float64).contiguous()
            if tuple(v.shape) != shape:
                raise ValueError("expected shape %s, got %s" % (shape, tuple(v.shape)))
            torch.cuda.current_stream().synchronize()
            check(L.bmg_field_set_level(g.ptr, self.scalar, lvl, v.data_ptr(), v.numel(),
                                        _lib.DEVICE), "bmg_field_set")
        else:
            if _is_torch(values):
                values = values.detach().cpu().numpy()
            v = np.asarray(values, dtype=np.float64)
            if v.ndim == 0:
                v = np.full(shape, float(v))
            v = np.ascontiguousarray(v)
            if v.shape != shape:
                raise ValueError("expected shape %s, got %s" % (shape, v.shape))
            check(L.bmg_field_set_level(g.ptr, self.scalar, lvl, v.ctypes.data, v.size,
                                        _lib.HOST), "bmg_field_set")
        return self

    def get(self, level=None, out=None):
        """Values of the finest level (or of ``level``) as a numpy array, or
        into ``out`` (a CUDA torch tensor, written on the device)."""
        g = self.grid
        lvl = g.depth if level is None else level
        shape = self.shape(lvl)
        L = _lib.load()
        if out is not None and _is_torch(out) and out.is_cuda:
            import torch
            assert out.dtype == torch.float64 and out.is_contiguous() and tuple(out.shape) == shape
            torch.cuda.current_stream().synchronize()
            check(L.bmg_field_get_level(g.ptr, self.scalar, lvl, out.data_ptr(), out.numel(),
                                        _lib.DEVICE), "bmg_field_get")
            return out
        v = np.empty(shape, dtype=np.float64)
        check(L.bmg_field_get_level(g.ptr, self.scalar, lvl, v.ctypes.data, v.size, _lib.HOST),
              "bmg_field_get")
        return v

    def bc(self, side, kind, value=0.0, values=None):
        """``s[side] = dirichlet(value)`` / ``neumann(value)`` (common.h:957-960);
        ``values``: one value per boundary face of the finest level."""
        g = self.grid
        L = _lib.load()
        kind = KINDS[kind] if isinstance(kind, str) else int(kind)
        if values is not None:
            if _is_torch(values) and values.is_cuda:
                v = values.detach().double().contiguous()
                check(L.bmg_bc(g.ptr, self.scalar, _side(side), kind, value, v.data_ptr(),
                               _lib.DEVICE), "bmg_bc")
                return self
            if _is_torch(values):
                values = values.detach().cpu().numpy()
            v = np.ascontiguousarray(values, dtype=np.float64).ravel()
            check(L.bmg_bc(g.ptr, self.scalar, _side(side), kind, value, v.ctypes.data,
                           _lib.HOST), "bmg_bc")
        else:
            check(L.bmg_bc(g.ptr, self.scalar, _side(side), kind, value, None, _lib.HOST),
                  "bmg_bc")
        return self

    def bc_level(self, side, kind, level, values):
        """``s[side] = dirichlet / neumann`` with the values of one level's
        boundary faces (a tree applies a field's conditions on every level)."""
        g = self.grid
        kind = KINDS[kind] if isinstance(kind, str) else int(kind)
        if _is_torch(values):
            values = values.detach().cpu().numpy()
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        check(_lib.load().bmg_bc_level(g.ptr, self.scalar, _side(side), kind, level,
                                       v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       _lib.HOST), "bmg_bc_level")
        return self


class Scalar(Field):
    pass


class FaceVector:
    def __init__(self, grid, handles, const=None):
        self.grid, self.const = grid, const
        self.components = [Field(grid, h, d, const) for d, h in enumerate(handles)]

    @property
    def vector(self):
        h = [c.handle for c in self.components] + [0] * (3 - len(self.components))
        return bmg_vector(bmg_scalar(h[0]), bmg_scalar(h[1]), bmg_scalar(h[2]))

    def set(self, comps, level=None):
        for c, v in zip(self.components, comps):
            c.set(v, level)
        return self

    def get(self, level=None):
        return [c.get(level) for c in self.components]


class Grid:
    """Levels 0..depth of a 2^depth-per-side box on the current CUDA device
    (``init_grid``, grid/multigrid.h:723-759).

    relax: ``"rbgs"`` (red-black Gauss-Seidel) or ``"jacobi"`` (the
    reference's -DJACOBI weighted Jacobi, poisson.h:293-328);
    precision: ``"fp64"`` or ``"mixed"`` (FP32 cycles inside FP64 iterative
    refinement).
    """

    def __init__(self, dim, depth, L0=1.0, origin=(0.0, 0.0, 0.0), relax="rbgs",
                 precision="fp64", graphs=True):
        L = _lib.load()
        self.dim, self.depth, self.n = dim, depth, 1 << depth
        p = ctypes.c_void_p()
        check(L.bmg_grid_new(ctypes.byref(p), dim, depth), "bmg_grid_new")
        self.ptr = p
        self.L0 = L0
        self.origin = tuple(origin) + (0.0,) * (3 - len(origin))
        check(L.bmg_size(self.ptr, L0), "bmg_size")
        check(L.bmg_origin(self.ptr, *self.origin[:3]), "bmg_origin")
        self.set_relax(relax)
        self.set_precision(precision)
        check(L.bmg_set_graphs(self.ptr, 1 if graphs else 0), "bmg_set_graphs")
        self._keep = []

    def close(self):
        if getattr(self, "ptr", None):
            _lib.load().bmg_grid_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- settings ----
    def set_relax(self, relax):
        r = {"rbgs": _lib.RELAX_RBGS, "jacobi": _lib.RELAX_JACOBI}.get(relax, relax)
        check(_lib.load().bmg_set_relax(self.ptr, r), "bmg_set_relax")

    def set_precision(self, precision):
        p = {"fp64": _lib.FP64, "mixed": _lib.MIXED}.get(precision, precision)
        check(_lib.load().bmg_set_precision(self.ptr, p), "bmg_set_precision")

    def set_graphs(self, n):
        """0/False: plain launches; 1/True: graphs with the default cache;
        n > 1: a cache of n captured V-cycles."""
        check(_lib.load().bmg_set_graphs(self.ptr, int(n)), "bmg_set_graphs")

    def set_timing(self, on):
        check(_lib.load().bmg_set_timing(self.ptr, 1 if on else 0), "bmg_set_timing")

    def set_stream(self, stream_ptr):
        check(_lib.load().bmg_set_stream(self.ptr, stream_ptr), "bmg_set_stream")

    def periodic(self, side):
        """``periodic(right)`` (cartesian-common.h:920-933)."""
        check(_lib.load().bmg_periodic(self.ptr, _side(side)), "bmg_periodic")

    def select(self):
        check(_lib.load().bmg_grid_select(self.ptr), "bmg_grid_select")

    def synchronize(self):
        check(_lib.load().bmg_synchronize(self.ptr), "bmg_synchronize")

    @property
    def delta(self):
        return self.L0 * (1.0 / (1 << self.depth))

    # ---- fields ----
    def scalar(self, values=None):
        s = bmg_scalar()
        check(_lib.load().bmg_scalar_new(self.ptr, ctypes.byref(s)), "bmg_scalar_new")
        f = Scalar(self, s.i)
        if values is not None:
            f.set(values)
        return f

    def face_vector(self, comps=None):
        v = bmg_vector()
        check(_lib.load().bmg_face_vector_new(self.ptr, ctypes.byref(v)), "bmg_face_vector_new")
        fv = FaceVector(self, [v.x.i, v.y.i, v.z.i][:self.dim])
        if comps is not None:
            fv.set(comps)
        return fv

    def const_scalar(self, value):
        s = bmg_scalar()
        check(_lib.load().bmg_const_scalar(self.ptr, value, ctypes.byref(s)), "bmg_const_scalar")
        return Scalar(self, s.i, const=value)

    def const_face_vector(self, value):
        v = bmg_vector()
        check(_lib.load().bmg_const_face_vector(self.ptr, value, ctypes.byref(v)),
              "bmg_const_face_vector")
        return FaceVector(self, [v.x.i, v.y.i, v.z.i][:self.dim], const=value)

    def delete(self, field):
        check(_lib.load().bmg_field_delete(self.ptr, field.scalar), "bmg_field_delete")

    # ---- the solver ----
    def _poisson_struct(self, a, b, alpha, lambda_, tolerance, nrelax, minlevel, res):
        p = _lib.Poisson()
        p.a, p.b = a.scalar, b.scalar
        if alpha is not None:
            p.alpha = alpha.vector
        if lambda_ is not None:
            p.lambda_ = lambda_.scalar
        p.tolerance, p.nrelax, p.minlevel = tolerance, nrelax, minlevel
        if res is not None:
            arr = (bmg_scalar * 2)(res.scalar, bmg_scalar(0))
            self._keep.append(arr)
            p.res = ctypes.cast(arr, ctypes.POINTER(bmg_scalar))
        return p

    def poisson(self, a, b, alpha=None, lambda_=None, tolerance=0.0, nrelax=0, minlevel=0,
                res=None, check_status=True):
        """``poisson (a, b, alpha, lambda, tolerance, nrelax, minlevel, res)``
        (poisson.h:402-441); returns mgstats as a dict (plus ``status``)."""
        L = _lib.load()
        p = self._poisson_struct(a, b, alpha, lambda_, tolerance, nrelax, minlevel, res)
        st = _lib.mgstats()
        status = L.bmg_poisson(self.ptr, p, ctypes.byref(st))
        if check_status and status not in (_lib.OK, _lib.ENOTCONV):
            check(status, "bmg_poisson")
        d = st.as_dict()
        d["status"] = status
        return d

    def vector(self, comps=None):
        """A cell-centred vector: one scalar per dimension (``vector u[]``)."""
        return [self.scalar(None if comps is None else comps[d]) for d in range(self.dim)]

    def viscosity(self, u, mu, rho, dt, nrelax=0, res=None):
        """``viscosity (u, mu, rho, dt, nrelax, res)`` (viscosity.h:169-183):
        u a list of dim cell scalars, mu a FaceVector (constant allowed), rho
        a Scalar (constant allowed); returns mgstats as a dict (plus
        ``status``)."""
        L = _lib.load()
        q = _lib.Viscosity()
        hs = [c.handle for c in u] + [0] * (3 - len(u))
        q.u = bmg_vector(bmg_scalar(hs[0]), bmg_scalar(hs[1]), bmg_scalar(hs[2]))
        q.mu, q.rho = mu.vector, rho.scalar
        q.dt, q.nrelax = dt, nrelax
        if res is not None:
            arr = (bmg_scalar * (len(res) + 1))(*[r.scalar for r in res], bmg_scalar(0))
            self._keep.append(arr)
            q.res = ctypes.cast(arr, ctypes.POINTER(bmg_scalar))
        st = _lib.mgstats()
        status = L.bmg_viscosity(self.ptr, q, ctypes.byref(st))
        if status not in (_lib.OK, _lib.ENOTCONV):
            check(status, "bmg_viscosity")
        d = st.as_dict()
        d["status"] = status
        return d

    def project(self, uf, p, alpha=None, dt=0.0, nrelax=0):
        """``project (uf, p, alpha, dt, nrelax)`` (poisson.h:468-509): makes
        the face vector uf discretely divergence-free with the pressure p;
        returns the mgstats of the pressure solve as a dict (plus ``status``)."""
        L = _lib.load()
        q = _lib.Project()
        q.uf, q.p = uf.vector, p.scalar
        if alpha is not None:
            q.alpha = alpha.vector
        q.dt, q.nrelax = dt, nrelax
        st = _lib.mgstats()
        status = L.bmg_project(self.ptr, q, ctypes.byref(st))
        if status not in (_lib.OK, _lib.ENOTCONV):
            check(status, "bmg_project")
        d = st.as_dict()
        d["status"] = status
        return d

    def mg_solve(self, a, b, alpha=None, lambda_=None, tolerance=0.0, nrelax=0, minlevel=0,
                 res=None):
        """``mg_solve`` (poisson.h:139-235) with the Poisson callbacks; unlike
        poisson() it does not restrict the coefficients first."""
        L = _lib.load()
        self.select()
        p = self._poisson_struct(a, b, alpha, lambda_, 0.0, nrelax, minlevel, None)
        al = (bmg_scalar * 2)(a.scalar, bmg_scalar(0))
        bl = (bmg_scalar * 2)(b.scalar, bmg_scalar(0))
        m = _lib.MGSolve()
        m.a = ctypes.cast(al, ctypes.POINTER(bmg_scalar))
        m.b = ctypes.cast(bl, ctypes.POINTER(bmg_scalar))
        m.residual = ctypes.cast(L.bmg_residual, ctypes.c_void_p)
        m.relax = ctypes.cast(L.bmg_relax, ctypes.c_void_p)
        m.data = ctypes.cast(ctypes.pointer(p), ctypes.c_void_p)
        m.nrelax, m.minlevel, m.tolerance = nrelax, minlevel, tolerance
        if res is not None:
            rl = (bmg_scalar * 2)(res.scalar, bmg_scalar(0))
            m.res = ctypes.cast(rl, ctypes.POINTER(bmg_scalar))
        st = L.mg_solve(m)
        status = L.bmg_last_error()
        if status not in (_lib.OK, _lib.ENOTCONV):
            check(status, "mg_solve")
        d = st.as_dict()
        d["status"] = status
        return d

    def residual(self, a, b, res, alpha=None, lambda_=None):
        """``residual (a, b, res, data)`` (poisson.h:345-391): writes res and
        returns max |res|."""
        L = _lib.load()
        self.select()
        p = self._poisson_struct(a, b, alpha, lambda_, 0.0, 0, 0, None)
        al = (bmg_scalar * 1)(a.scalar)
        bl = (bmg_scalar * 1)(b.scalar)
        rl = (bmg_scalar * 1)(res.scalar)
        m = L.bmg_residual(al, bl, rl, ctypes.cast(ctypes.pointer(p), ctypes.c_void_p))
        check(L.bmg_last_error(), "bmg_residual")
        return m

    def mg_cycle(self, a, res, da, nrelax, minlevel, maxlevel, alpha=None, lambda_=None):
        """``mg_cycle (a, res, da, relax, data, nrelax, minlevel, maxlevel)``
        (poisson.h:32-90) with the Poisson relax."""
        L = _lib.load()
        self.select()
        p = self._poisson_struct(a, a, alpha, lambda_, 0.0, 0, 0, None)
        al = (bmg_scalar * 1)(a.scalar)
        rl = (bmg_scalar * 1)(res.scalar)
        dl = (bmg_scalar * 1)(da.scalar)
        L.mg_cycle(al, rl, dl, ctypes.cast(L.bmg_relax, ctypes.c_void_p),
                   ctypes.cast(ctypes.pointer(p), ctypes.c_void_p), nrelax, minlevel, maxlevel)
        check(L.bmg_last_error(), "mg_cycle")

    def restriction(self, fields):
        """restriction (list) (multigrid-common.h:368-404)."""
        hs = []
        for f in fields:
            if isinstance(f, FaceVector):
                hs.append(f.components[0].handle)
            else:
                hs.append(f.handle)
        arr = (bmg_scalar * (len(hs) + 1))(*[bmg_scalar(h) for h in hs], bmg_scalar(0))
        check(_lib.load().bmg_restriction(self.ptr, arr), "bmg_restriction")

    def _named_list(self, fields):
        items = list(fields.items()) if isinstance(fields, dict) else list(fields)
        for name, f in items:
            if not isinstance(f, Field):
                raise TypeError("dump/restore take cell fields (%s)" % name)
        arr = (bmg_scalar * (len(items) + 1))(*[bmg_scalar(f.handle) for _, f in items],
                                              bmg_scalar(0))
        names = (ctypes.c_char_p * max(1, len(items)))(*[n.encode() for n, _ in items])
        return arr, names

    def dump(self, file, fields, t=0.0, i=0):
        """``dump (file, list)`` (output.h:1138-1171): fields is a dict (or
        list of pairs) name -> cell field; t and i go into the header."""
        arr, names = self._named_list(fields)
        check(_lib.load().bmg_dump(self.ptr, os.fsencode(file), arr, names, float(t), int(i)),
              "bmg_dump")

    def restore(self, file, fields):
        """``restore (file, list)`` (output.h:1220-1400): fills the fields
        whose names the file holds; returns the header's (t, i)."""
        arr, names = self._named_list(fields)
        t, i = ctypes.c_double(0.0), ctypes.c_int(0)
        check(_lib.load().bmg_restore(self.ptr, os.fsencode(file), arr, names,
                                      ctypes.byref(t), ctypes.byref(i)), "bmg_restore")
        # the file's origin and size now hold (output.h:1325-1326)
        with open(file, "rb") as fp:
            head = fp.read(56)
            nlen, version = ctypes.c_long.from_buffer_copy(head, 8).value, \
                ctypes.c_int.from_buffer_copy(head, 28).value
            if version != 161020:
                for _ in range(nlen):
                    fp.seek(ctypes.c_uint.from_buffer_copy(fp.read(4)).value, 1)
            o = np.frombuffer(fp.read(32), dtype=np.float64)
        self.origin, self.L0 = (float(o[0]), float(o[1]), float(o[2])), float(o[3])
        return t.value, i.value

    def counters(self):
        c = _lib.bmg_counters()
        check(_lib.load().bmg_get_counters(self.ptr, ctypes.byref(c)), "bmg_get_counters")
        return {k: getattr(c, k) for k, _ in c._fields_}

    def reset_counters(self):
        check(_lib.load().bmg_reset_counters(self.ptr), "bmg_reset_counters")


def set_tolerance(value):
    """The global TOLERANCE (poisson.h:103)."""
    _lib.global_var("TOLERANCE").value = value


def get_tolerance():
    return _lib.global_var("TOLERANCE").value


def set_niter(nitermax=None, nitermin=None):
    if nitermax is not None:
        _lib.global_var("NITERMAX").value = nitermax
    if nitermin is not None:
        _lib.global_var("NITERMIN").value = nitermin


class TreeGrid(Grid):
    """A quadtree (grid/quadtree.h) over the levels of a two-dimensional grid
    of depth ``maxdepth``: ``init_grid (1)`` then ``refine (cond)``.

    Field values live in the level arrays (``Field.set(values, level=l)`` /
    ``get(level=l)``); the solver reads the leaves, whose mask
    ``leaf_mask(l)`` gives.  ``poisson``, ``mg_solve``, ``mg_cycle``,
    ``residual`` and ``restriction`` follow the reference's tree branch.
    ``precision="mixed"`` runs the solve's cycles in FP32 inside FP64
    iterative refinement (the residual, a and b stay FP64).
    """

    def __init__(self, maxdepth, L0=1.0, origin=(0.0, 0.0), relax="rbgs", graphs=True,
                 precision="fp64"):
        super().__init__(2, maxdepth, L0=L0, origin=origin, relax=relax, precision=precision,
                         graphs=graphs)
        self.maxdepth = maxdepth

    def refine(self, cond):
        """``refine (cond)`` (tree-common.h:308-326) with ``cond(level, x, y)``
        evaluated at leaf centres; returns the number of refined cells."""
        cb = _lib.REFINE_COND(lambda l, x, y, z, d: 1 if cond(l, x, y) else 0)
        r = _lib.load().bmg_tree_refine(self.ptr, cb, None)
        if r < 0:
            check(r, "bmg_tree_refine")
        return r

    def restore(self, file, fields):
        """``restore (file, list)`` on a tree: init_grid (1), then the file's
        refinement (output.h:1237-1242, 1357-1358)."""
        if not self._has_tree():
            self.refine(lambda l, x, y: False)
        return super().restore(file, fields)

    def _has_tree(self):
        return _lib.load().bmg_tree_info(self.ptr, None, None) == _lib.OK

    def info(self):
        d = ctypes.c_int()
        n = ctypes.c_longlong()
        check(_lib.load().bmg_tree_info(self.ptr, ctypes.byref(d), ctypes.byref(n)),
              "bmg_tree_info")
        return d.value, n.value

    @property
    def tree_depth(self):
        return self.info()[0]

    @property
    def leaves(self):
        return self.info()[1]

    def flags(self, level):
        n = 1 << level
        out = np.zeros((n, n), dtype=np.uint8)
        check(_lib.load().bmg_tree_flags(self.ptr, level,
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))),
              "bmg_tree_flags")
        return out

    def leaf_mask(self, level):
        return (self.flags(level) & _lib.TREE_LEAF) != 0

    def level_delta(self, level):
        return self.L0 * (1.0 / (1 << level))

    def centers(self, level):
        """Cell centres of one level, ``x = (i + 0.5) Delta + X0``."""
        n = 1 << level
        c = (np.arange(n) + 0.5) * self.level_delta(level)
        return np.meshgrid(c + self.origin[0], c + self.origin[1], indexing="ij")
