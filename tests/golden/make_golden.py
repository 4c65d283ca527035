"""Collect the reference's golden logs for the Poisson path into a fixture.

Reads the Basilisk test logs (``src/test/*.ref``, ``*.cref``) from the
``src`` directory of a reference checkout, given as argv[1] or in the
environment variable BASILISK_SRC, and writes ``reference_logs.json`` next
to this script.  The logs are the reference's own known-answer outputs; the drivers
in ``tests/golden_drivers.py`` reproduce the programs that printed them.
Run once; the committed JSON is what the tests read.
"""
import json
import os
import sys

LOGS = {
    # program (reference file)          -> log file(s) it is pinned by
    "poisson_2d":   ("test/poisson.c", "test/poisson.cref"),
    "poisson_2d_quadtree": ("test/poisson.c", "test/poisson.ref"),
    "poisson_3d":   ("test/poisson.c", "test/poisson.3D.ref"),
    "variable_2d":  ("test/variable.c", "test/variable.ref"),
    "periodic_2d":  ("test/periodic.c", "test/periodic.ref"),
    "periodic_3d":  ("test/periodic.c", "test/periodic.3D.ref"),
    "poisson_1d":   ("test/poisson1D.c", "test/poisson1D.ref"),
    "circle_2d":    ("test/circle.c", "test/circle.ref"),
    "circle_variable_2d": ("test/circle-variable.c", "test/circle-variable.ref"),
    "solenoidal_2d": ("test/solenoidal.c", "test/solenoidal.ref"),
}


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BASILISK_SRC")
    if not root:
        sys.exit("usage: make_golden.py <basilisk checkout>/src  (or set BASILISK_SRC)")
    out = {}
    for key, (prog, log) in LOGS.items():
        with open(os.path.join(root, log)) as f:
            out[key] = {"program": prog, "log": log,
                        "lines": f.read().splitlines()}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_logs.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
