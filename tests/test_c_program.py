"""The C-ABI as a C caller sees it: a C99 program written against
include/basilisk_mg.h compiles with warnings as errors, links against
libbmg.so and runs.  Without a device every entry point reports BMG_ENODEV
(there is no CPU fallback); with one, the program solves a small Poisson
problem through poisson () as the reference's test programs do."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "basilisk_b200")

PROGRAM = r"""
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "basilisk_mg.h"

int main (void)
{
  bmg_grid * g = NULL;
  int r = bmg_grid_new (&g, 2, 5);           /* init_grid (32) */
  if (r == BMG_ENODEV) {
    printf ("nodev %s\n", bmg_error_string (bmg_last_error ()));
    return 0;
  }
  if (r != BMG_OK) return 2;
  const int n = 32;
  bmg_scalar a, b;
  bmg_vector alpha;
  if (bmg_scalar_new (g, &a) || bmg_scalar_new (g, &b) || bmg_face_vector_new (g, &alpha))
    return 3;
  for (int side = BMG_RIGHT; side <= BMG_BOTTOM; side++)
    if (bmg_bc (g, a, side, BMG_DIRICHLET, 0., NULL, BMG_HOST)) return 4;
  double * rhs = malloc (n*n*sizeof (double)), * ax = malloc ((n + 1)*n*sizeof (double));
  for (int k = 0; k < n*n; k++) rhs[k] = sin (0.1*k);
  for (int k = 0; k < (n + 1)*n; k++) ax[k] = 1. + 0.5*cos (0.2*k);
  if (bmg_field_set (g, b, rhs, n*n, BMG_HOST) ||
      bmg_field_set (g, alpha.x, ax, (n + 1)*n, BMG_HOST) ||
      bmg_field_set (g, alpha.y, ax, n*(n + 1), BMG_HOST)) return 5;
  mgstats s = poisson ((struct Poisson){a, b, alpha, .tolerance = 1e-8});
  if (bmg_last_error () != BMG_OK || !(s.resa <= 1e-8) || s.i < 1) return 6;
  bmg_field_get (g, a, rhs, n*n, BMG_HOST);
  bmg_grid_free (g);
  printf ("solved %d %g\n", s.i, s.resa);
  free (rhs); free (ax);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_against_the_header(tmp_path):
    if not os.path.exists(os.path.join(LIB, "libbmg.so")):
        pytest.skip("libbmg.so is not built")
    src = tmp_path / "prog.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "prog"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-o", str(exe), str(src),
                    "-I", os.path.join(ROOT, "include"), "-L", LIB, "-lbmg",
                    "-Wl,-rpath," + LIB, "-lm"], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.startswith("nodev") or out.stdout.startswith("solved"), out.stdout
