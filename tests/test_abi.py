"""The C-ABI library: it loads without a GPU, exports every symbol that
include/basilisk_mg.h declares, keeps the reference's struct layouts and
globals, and fails with a status (never a crash) when no device exists."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import HAS_GPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "basilisk_mg.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    # typedefs of function-pointer types declare no symbol
    text = re.sub(r"^\s*typedef[^;]*;", "", text, flags=re.M | re.S)
    names = set()
    for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
        name = m.group(1)
        if name not in ("if", "while", "for", "return", "sizeof"):
            names.add(name)
    # function-pointer members of struct MGSolve are not exported symbols
    names -= {"residual", "relax"}
    return sorted(names)


def test_library_loads_and_exports_everything():
    from basilisk_b200 import _lib
    L = _lib.load()
    names = declared_functions()
    assert "poisson" in names and "mg_solve" in names and "mg_cycle" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the binding declares exactly the header's functions
    assert set(_lib.SIGNATURES) == set(names)


def test_globals_have_reference_defaults():
    from basilisk_b200 import _lib
    assert _lib.global_var("NITERMAX").value == 100
    assert _lib.global_var("NITERMIN").value == 1
    assert _lib.global_var("TOLERANCE").value == 1e-3


def test_struct_layouts_match_header(tmp_path):
    """Offsets of mgstats / struct Poisson / struct MGSolve as compiled from
    the header equal the ctypes mirrors (and mgstats is the reference's
    {int; double; double; double; int; int})."""
    from basilisk_b200 import _lib
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "basilisk_mg.h"
int main (void) {
  printf ("%zu %zu %zu %zu %zu %zu %zu\n", sizeof (mgstats), offsetof (mgstats, i),
          offsetof (mgstats, resb), offsetof (mgstats, resa), offsetof (mgstats, sum),
          offsetof (mgstats, nrelax), offsetof (mgstats, minlevel));
  printf ("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof (struct Poisson),
          offsetof (struct Poisson, a), offsetof (struct Poisson, b),
          offsetof (struct Poisson, alpha), offsetof (struct Poisson, lambda),
          offsetof (struct Poisson, tolerance), offsetof (struct Poisson, nrelax),
          offsetof (struct Poisson, minlevel), offsetof (struct Poisson, res));
  printf ("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof (struct MGSolve),
          offsetof (struct MGSolve, a), offsetof (struct MGSolve, b),
          offsetof (struct MGSolve, residual), offsetof (struct MGSolve, relax),
          offsetof (struct MGSolve, data), offsetof (struct MGSolve, nrelax),
          offsetof (struct MGSolve, res), offsetof (struct MGSolve, minlevel),
          offsetof (struct MGSolve, tolerance));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    m = [int(x) for x in out[0].split()]
    S = _lib.mgstats
    assert m == [ctypes.sizeof(S), S.i.offset, S.resb.offset, S.resa.offset, S.sum.offset,
                 S.nrelax.offset, S.minlevel.offset]
    assert m == [40, 0, 8, 16, 24, 32, 36]
    p = [int(x) for x in out[1].split()]
    Pz = _lib.Poisson
    assert p == [ctypes.sizeof(Pz), Pz.a.offset, Pz.b.offset, Pz.alpha.offset,
                 Pz.lambda_.offset, Pz.tolerance.offset, Pz.nrelax.offset,
                 Pz.minlevel.offset, Pz.res.offset]
    q = [int(x) for x in out[2].split()]
    M = _lib.MGSolve
    assert q == [ctypes.sizeof(M), M.a.offset, M.b.offset, M.residual.offset, M.relax.offset,
                 M.data.offset, M.nrelax.offset, M.res.offset, M.minlevel.offset,
                 M.tolerance.offset]


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_no_device_fails_with_status():
    from basilisk_b200 import _lib
    L = _lib.load()
    p = ctypes.c_void_p()
    assert L.bmg_grid_new(ctypes.byref(p), 2, 5) == _lib.ENODEV
    assert L.bmg_last_error() == _lib.ENODEV
    # the reference-named entry point returns zeroed mgstats and a status
    st = L.poisson(_lib.Poisson())
    assert st.i == 0 and L.bmg_last_error() == _lib.EINVAL
    with pytest.raises(_lib.BMGError):
        import basilisk_b200
        basilisk_b200.Grid(2, 5)


def test_invalid_arguments_rejected():
    from basilisk_b200 import _lib
    L = _lib.load()
    p = ctypes.c_void_p()
    assert L.bmg_grid_new(ctypes.byref(p), 4, 5) == _lib.EINVAL
    assert L.bmg_grid_new(ctypes.byref(p), 2, -1) == _lib.EINVAL
    assert L.bmg_grid_new(None, 2, 3) == _lib.EINVAL
    st = _lib.mgstats()
    assert L.bmg_poisson(None, _lib.Poisson(), ctypes.byref(st)) == _lib.EINVAL
