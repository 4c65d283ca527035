"""ctypes binding of ``libbmg.so`` (declared in ``include/basilisk_mg.h``).

The library is the product: a C host layer plus sm_100a CUDA kernels.  This
module only loads it and declares the signatures; it raises if the library
is missing or no CUDA device is present -- there is no fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libbmg.so")

# status codes
OK, EINVAL, ECUDA, ENOMEM, ENAN, ENOTCONV, EUNSUPPORTED, ENODEV = range(8)
# sides (common.h:949)
RIGHT, LEFT, TOP, BOTTOM, FRONT, BACK = range(6)
NEUMANN, DIRICHLET, PERIODIC = 0, 1, 2
RELAX_RBGS, RELAX_JACOBI = 0, 1
FP64, MIXED = 0, 1
HOST, DEVICE = 0, 1


class BMGError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = _lib.bmg_error_string(status).decode() if _lib else str(status)
        super().__init__("%s: %s (status %d)" % (what, msg, status))


class mgstats(ctypes.Structure):
    """``mgstats`` of poisson.h:108-114 (same members, same order)."""
    _fields_ = [("i", ctypes.c_int), ("resb", ctypes.c_double),
                ("resa", ctypes.c_double), ("sum", ctypes.c_double),
                ("nrelax", ctypes.c_int), ("minlevel", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class bmg_scalar(ctypes.Structure):
    _fields_ = [("i", ctypes.c_int)]


class bmg_vector(ctypes.Structure):
    _fields_ = [("x", bmg_scalar), ("y", bmg_scalar), ("z", bmg_scalar)]


class Poisson(ctypes.Structure):
    """``struct Poisson`` of poisson.h:258-265."""
    _fields_ = [("a", bmg_scalar), ("b", bmg_scalar), ("alpha", bmg_vector),
                ("lambda_", bmg_scalar), ("tolerance", ctypes.c_double),
                ("nrelax", ctypes.c_int), ("minlevel", ctypes.c_int),
                ("res", ctypes.POINTER(bmg_scalar))]


class Project(ctypes.Structure):
    """``struct Project`` of poisson.h:461-467."""
    _fields_ = [("uf", bmg_vector), ("p", bmg_scalar), ("alpha", bmg_vector),
                ("dt", ctypes.c_double), ("nrelax", ctypes.c_int)]


class Viscosity(ctypes.Structure):
    """``struct Viscosity`` of viscosity.h:3-10."""
    _fields_ = [("u", bmg_vector), ("mu", bmg_vector), ("rho", bmg_scalar),
                ("dt", ctypes.c_double), ("nrelax", ctypes.c_int),
                ("res", ctypes.POINTER(bmg_scalar))]


RELAX_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(bmg_scalar), ctypes.POINTER(bmg_scalar),
                            ctypes.c_int, ctypes.c_void_p)
# int (*) (int level, double x, double y, double z, void * data)
REFINE_COND = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, ctypes.c_void_p)
RESIDUAL_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.POINTER(bmg_scalar),
                               ctypes.POINTER(bmg_scalar), ctypes.POINTER(bmg_scalar),
                               ctypes.c_void_p)


class MGSolve(ctypes.Structure):
    """``struct MGSolve`` of poisson.h:125-137."""
    _fields_ = [("a", ctypes.POINTER(bmg_scalar)), ("b", ctypes.POINTER(bmg_scalar)),
                ("residual", ctypes.c_void_p), ("relax", ctypes.c_void_p),
                ("data", ctypes.c_void_p), ("nrelax", ctypes.c_int),
                ("res", ctypes.POINTER(bmg_scalar)), ("minlevel", ctypes.c_int),
                ("tolerance", ctypes.c_double)]


class bmg_counters(ctypes.Structure):
    _fields_ = [("cycles", ctypes.c_longlong), ("sweeps", ctypes.c_longlong),
                ("bytes", ctypes.c_double), ("cycle_ms", ctypes.c_double),
                ("launches", ctypes.c_longlong), ("relax_ms", ctypes.c_double),
                ("relax_bytes", ctypes.c_double), ("relax_sweeps", ctypes.c_longlong)]


# every function the header declares, with its signature
# flags of bmg_tree_flags (basilisk_mg.h)
TREE_ACTIVE, TREE_LEAF, TREE_HALO, TREE_PROLONGATION = 1, 2, 4, 8

P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
SZ = ctypes.c_size_t
DP = ctypes.c_void_p   # double * (host or device address)
SIGNATURES = {
    "bmg_error_string": (ctypes.c_char_p, [I]),
    "bmg_last_error": (I, []),
    "bmg_grid_new": (I, [ctypes.POINTER(P), I, I]),
    "bmg_grid_free": (None, [P]),
    "bmg_grid_select": (I, [P]),
    "bmg_grid_current": (P, []),
    "bmg_grid_info": (I, [P, ctypes.POINTER(I), ctypes.POINTER(I)]),
    "bmg_origin": (I, [P, D, D, D]),
    "bmg_size": (I, [P, D]),
    "bmg_periodic": (I, [P, I]),
    "bmg_set_relax": (I, [P, I]),
    "bmg_set_precision": (I, [P, I]),
    "bmg_set_stream": (I, [P, P]),
    "bmg_synchronize": (I, [P]),
    "bmg_scalar_new": (I, [P, ctypes.POINTER(bmg_scalar)]),
    "bmg_face_vector_new": (I, [P, ctypes.POINTER(bmg_vector)]),
    "bmg_const_scalar": (I, [P, D, ctypes.POINTER(bmg_scalar)]),
    "bmg_const_face_vector": (I, [P, D, ctypes.POINTER(bmg_vector)]),
    "bmg_field_delete": (I, [P, bmg_scalar]),
    "bmg_field_set": (I, [P, bmg_scalar, DP, SZ, I]),
    "bmg_field_get": (I, [P, bmg_scalar, DP, SZ, I]),
    "bmg_field_get_level": (I, [P, bmg_scalar, I, DP, SZ, I]),
    "bmg_field_set_level": (I, [P, bmg_scalar, I, DP, SZ, I]),
    "bmg_bc": (I, [P, bmg_scalar, I, I, D, DP, I]),
    "poisson": (mgstats, [Poisson]),
    "bmg_poisson": (I, [P, Poisson, ctypes.POINTER(mgstats)]),
    "project": (mgstats, [Project]),
    "viscosity": (mgstats, [Viscosity]),
    "bmg_viscosity": (I, [P, Viscosity, ctypes.POINTER(mgstats)]),
    "bmg_project": (I, [P, Project, ctypes.POINTER(mgstats)]),
    "bmg_relax": (None, [ctypes.POINTER(bmg_scalar), ctypes.POINTER(bmg_scalar), I, P]),
    "bmg_residual": (D, [ctypes.POINTER(bmg_scalar), ctypes.POINTER(bmg_scalar),
                         ctypes.POINTER(bmg_scalar), P]),
    "mg_solve": (mgstats, [MGSolve]),
    "mg_cycle": (None, [ctypes.POINTER(bmg_scalar), ctypes.POINTER(bmg_scalar),
                        ctypes.POINTER(bmg_scalar), P, P, I, I, I]),
    "bmg_restriction": (I, [P, ctypes.POINTER(bmg_scalar)]),
    "bmg_tree_refine": (I, [P, REFINE_COND, P]),
    "bmg_tree_info": (I, [P, ctypes.POINTER(I), ctypes.POINTER(ctypes.c_longlong)]),
    "bmg_tree_flags": (I, [P, I, ctypes.POINTER(ctypes.c_ubyte)]),
    "bmg_bc_level": (I, [P, bmg_scalar, I, I, I, DP, I]),
    "bmg_dump": (I, [P, ctypes.c_char_p, ctypes.POINTER(bmg_scalar),
                     ctypes.POINTER(ctypes.c_char_p), D, I]),
    "bmg_restore": (I, [P, ctypes.c_char_p, ctypes.POINTER(bmg_scalar),
                        ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(D),
                        ctypes.POINTER(I)]),
    "bmg_get_counters": (I, [P, ctypes.POINTER(bmg_counters)]),
    "bmg_reset_counters": (I, [P]),
    "bmg_set_timing": (I, [P, I]),
    "bmg_set_graphs": (I, [P, I]),
    "bmg_sum_noalloc": (I, [P, SZ, P, P]),
    "bmg_shard_new": (I, [ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(I),
                          ctypes.POINTER(I)]),
    "bmg_shard_free": (None, [P]),
    "bmg_shard_poisson": (I, [P, Poisson, ctypes.POINTER(mgstats)]),
    "bmg_shard_dims": (I, [I, I, ctypes.POINTER(I)]),
    "bmg_shard_neighbours": (I, [I, ctypes.POINTER(I), ctypes.POINTER(I), I,
                                 ctypes.POINTER(I)]),
    "bmg_adjoint_gradients": (I, [P, bmg_scalar, bmg_scalar, ctypes.POINTER(P), P, I]),
}
GLOBALS = {"NITERMAX": ctypes.c_int, "NITERMIN": ctypes.c_int, "TOLERANCE": ctypes.c_double}

_lib = None


def load(path=LIBPATH):
    """Load libbmg.so and declare its signatures (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libbmg.so is not built (%s); run __graft_entry__.build() "
                          "or make -C basilisk_b200/csrc" % path)
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status, what=""):
    if status != OK:
        raise BMGError(status, what)


def global_var(name):
    return GLOBALS[name].in_dll(load(), name)
