"""A domain decomposed into blocks, the counterpart of Basilisk's
``grid/multigrid-mpi.h`` over the C-ABI of ``libbmg.so``.

The reference runs one multigrid hierarchy per MPI rank on a
``dims[0] x dims[1] (x dims[2])`` Cartesian arrangement of blocks
(``MPI_Dims_create`` / ``MPI_Cart_create``, multigrid-mpi.h:94-130) and
exchanges the ghost layers of neighbouring blocks after every boundary
(``mpi_boundary_level``, multigrid-mpi.h:52-85).  Here each block is a
``Grid`` on a CUDA device (several blocks may share a device) and one
``bmg_shard_poisson`` call runs the whole decomposed solve: the exchanges
are device (or peer) copies, the reductions happen over the blocks.

Global arrays are given and returned in the layout of one grid covering the
whole domain: ``dims[e] * 2**depth`` cells along direction ``e`` (plus one
face along a face vector's own direction); ``set`` scatters them into the
blocks, ``get`` gathers them.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check
from .grid import Grid, KINDS, _side, _is_torch


def dims_create(n, dim):
    """``MPI_Dims_create (n, dim, dims)`` with all dims free."""
    d = (ctypes.c_int * 3)()
    check(_lib.load().bmg_shard_dims(n, dim, d), "bmg_shard_dims")
    return tuple(d[:dim])


def neighbours(dim, dims, periodic, b):
    """``MPI_Cart_shift`` of block ``b``: the neighbouring block on each side
    (right, left, top, bottom, front, back), -1 on a box side."""
    d = (ctypes.c_int * 3)(*(list(dims) + [1] * (3 - len(dims))))
    p = (ctypes.c_int * 3)(*[1 if e in periodic else 0 for e in range(3)])
    out = (ctypes.c_int * 6)()
    check(_lib.load().bmg_shard_neighbours(dim, d, p, b, out), "bmg_shard_neighbours")
    return tuple(out[:2 * dim])


def _numpy(values):
    if _is_torch(values):
        values = values.detach().cpu().numpy()
    return np.asarray(values, dtype=np.float64)


class ShardedField:
    """One field of every block (the same handle in each)."""

    def __init__(self, sg, fields, face_dim=-1):
        self.sg, self.fields, self.face_dim = sg, fields, face_dim

    @property
    def scalar(self):
        return self.fields[0].scalar

    def _slices(self, b):
        n = self.sg.n
        c = self.sg.coords(b)
        return tuple(slice(c[e] * n, c[e] * n + n + (1 if e == self.face_dim else 0))
                     for e in range(self.sg.dim))

    def shape(self):
        n = self.sg.n
        return tuple(self.sg.dims[e] * n + (1 if e == self.face_dim else 0)
                     for e in range(self.sg.dim))

    def set(self, values):
        v = _numpy(values)
        if v.ndim == 0:
            v = np.full(self.shape(), float(v))
        if v.shape != self.shape():
            raise ValueError("expected shape %s, got %s" % (self.shape(), v.shape))
        for b, f in enumerate(self.fields):
            f.set(np.ascontiguousarray(v[self._slices(b)]))
        return self

    def get(self):
        out = np.empty(self.shape())
        for b, f in enumerate(self.fields):
            out[self._slices(b)] = f.get()
        return out

    def bc(self, side, kind, value=0.0, values=None):
        """``s[side] = dirichlet / neumann`` on the domain's side: a constant,
        or one value per boundary face of the whole side (the tangential
        indices in increasing dimension order), each block taking its part."""
        s = _side(side)
        e = s // 2
        n = self.sg.n
        for b, f in enumerate(self.fields):
            if values is None:
                f.bc(s, kind, value)
                continue
            tang = [d for d in range(self.sg.dim) if d != e]
            v = _numpy(values).reshape([self.sg.dims[d] * n for d in tang])
            c = self.sg.coords(b)
            part = v[tuple(slice(c[d] * n, c[d] * n + n) for d in tang)]
            f.bc(s, kind, value, np.ascontiguousarray(part))
        return self


class ShardedFaceVector:
    def __init__(self, sg, comps):
        self.sg, self.components = sg, comps

    @property
    def vector(self):
        return self._vector()

    def _vector(self):
        h = [c.fields[0].handle for c in self.components] + [0] * (3 - len(self.components))
        return _lib.bmg_vector(_lib.bmg_scalar(h[0]), _lib.bmg_scalar(h[1]),
                               _lib.bmg_scalar(h[2]))

    def set(self, comps):
        for c, v in zip(self.components, comps):
            c.set(v)
        return self

    def get(self):
        return [c.get() for c in self.components]


class ShardedGrid:
    """A domain of ``dims`` blocks of ``2**depth`` cells per side each.

    dims: the block arrangement (default ``dims_create(nblocks, dim)``);
    L0: the domain's extent along x (each block is ``L0 / dims[0]`` wide, as
    the reference rescales its resolution, multigrid-mpi.h:115-123);
    periodic: the periodic directions (0, 1, 2) of the domain;
    devices: the CUDA device of each block (default: all on the current
    one).  The solve is FP64; relax is ``"rbgs"`` or ``"jacobi"``.
    """

    def __init__(self, dim, depth, dims=None, nblocks=None, L0=1.0, origin=(0.0, 0.0, 0.0),
                 periodic=(), relax="rbgs", devices=None):
        if dims is None:
            dims = dims_create(nblocks or 1, dim)
        self.dim, self.depth, self.n = dim, depth, 1 << depth
        self.dims = tuple(dims)[:dim]
        self.periodic = tuple(sorted(set(periodic)))
        self.nb = int(np.prod(self.dims))
        bsize = L0 / self.dims[0]
        origin = tuple(origin) + (0.0,) * (3 - len(origin))
        self.blocks = []
        for b in range(self.nb):
            c = self.coords(b)
            org = [origin[e] + (c[e] * bsize if e < dim else 0.0) for e in range(3)]
            dev = None if devices is None else devices[b % len(devices)]
            if dev is not None:
                import torch
                with torch.cuda.device(dev):
                    g = Grid(dim, depth, L0=bsize, origin=org, relax=relax)
            else:
                g = Grid(dim, depth, L0=bsize, origin=org, relax=relax)
            for e in self.periodic:
                if self.dims[e] == 1:
                    g.periodic(2 * e)
            self.blocks.append(g)
        arr = (ctypes.c_void_p * self.nb)(*[g.ptr.value for g in self.blocks])
        d = (ctypes.c_int * 3)(*(list(self.dims) + [1] * (3 - dim)))
        p = (ctypes.c_int * 3)(*[1 if e in self.periodic else 0 for e in range(3)])
        ptr = ctypes.c_void_p()
        check(_lib.load().bmg_shard_new(ctypes.byref(ptr), arr, d, p), "bmg_shard_new")
        self.ptr = ptr

    def coords(self, b):
        """Cartesian coordinates of block ``b`` (row-major, as MPI_Cart_create)."""
        d = list(self.dims) + [1] * (3 - self.dim)
        c = (b // (d[1] * d[2]), (b // d[2]) % d[1], b % d[2])
        return c[:self.dim]

    def close(self):
        if getattr(self, "ptr", None):
            _lib.load().bmg_shard_free(self.ptr)
            self.ptr = None
        for g in getattr(self, "blocks", []):
            g.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def scalar(self, values=None):
        f = ShardedField(self, [g.scalar() for g in self.blocks])
        hs = {x.handle for x in f.fields}
        assert len(hs) == 1, "blocks gave different handles"
        if values is not None:
            f.set(values)
        return f

    def face_vector(self, comps=None):
        vs = [g.face_vector() for g in self.blocks]
        fv = ShardedFaceVector(self, [ShardedField(self, [v.components[d] for v in vs], d)
                                      for d in range(self.dim)])
        if comps is not None:
            fv.set(comps)
        return fv

    def const_scalar(self, value):
        return ShardedField(self, [g.const_scalar(value) for g in self.blocks])

    def poisson(self, a, b, alpha=None, lambda_=None, tolerance=0.0, nrelax=0, minlevel=0,
                res=None, check_status=True):
        """``poisson ()`` over the blocks (bmg_shard_poisson); returns mgstats
        as a dict (plus ``status``)."""
        p = _lib.Poisson()
        p.a, p.b = a.scalar, b.scalar
        if alpha is not None:
            p.alpha = alpha._vector()
        if lambda_ is not None:
            p.lambda_ = lambda_.scalar
        p.tolerance, p.nrelax, p.minlevel = tolerance, nrelax, minlevel
        keep = None
        if res is not None:
            keep = (_lib.bmg_scalar * 2)(res.scalar, _lib.bmg_scalar(0))
            p.res = ctypes.cast(keep, ctypes.POINTER(_lib.bmg_scalar))
        st = _lib.mgstats()
        status = _lib.load().bmg_shard_poisson(self.ptr, p, ctypes.byref(st))
        if check_status and status not in (_lib.OK, _lib.ENOTCONV):
            check(status, "bmg_shard_poisson")
        d = st.as_dict()
        d["status"] = status
        del keep
        return d


__all__ = ["ShardedGrid", "dims_create", "neighbours", "KINDS"]
