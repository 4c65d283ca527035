"""basilisk_b200 -- a B200-native multigrid Poisson--Helmholtz solver.

A from-scratch sm_100a implementation of Basilisk's multigrid
Poisson--Helmholtz solver (poisson.h mg_solve / mg_cycle with its relax and
residual stencils on grid/multigrid.h levels) behind a C-ABI
(``include/basilisk_mg.h``, ``libbmg.so``).  This package is the Python side
of that ABI: the grid/field front end (``Grid``), the reference's Python
``poisson()`` entry point, and the differentiable solve (``autograd``).
"""
from . import _lib
from ._lib import BMGError, load
from .grid import Grid, TreeGrid, Scalar, FaceVector, set_tolerance, get_tolerance, set_niter
from ._build import build


def poisson(a, b, alpha=None, lambda0=None, tolerance=1e-3, nrelax=0, minlevel=0):
    """The reference's Python entry point (poisson.i: ``poisson(a, b,
    alpha=None, lambda0=0, tolerance=1e-3)``) on the fields' grid."""
    return a.grid.poisson(a, b, alpha=alpha, lambda_=lambda0, tolerance=tolerance,
                          nrelax=nrelax, minlevel=minlevel)


__all__ = ["Grid", "TreeGrid", "Scalar", "FaceVector", "poisson", "build", "load", "BMGError",
           "set_tolerance", "get_tolerance", "set_niter"]
