"""Build ``libbmg.so`` in-tree (nvcc for sm_100a + gcc for the C host)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose=False):
    """Compile the CUDA kernels and the C host layer into basilisk_b200/libbmg.so."""
    out = subprocess.run(["make", "-C", os.path.join(HERE, "csrc")],
                         capture_output=True, text=True)
    if verbose or out.returncode != 0:
        print(out.stdout)
        print(out.stderr)
    if out.returncode != 0:
        raise RuntimeError("building libbmg.so failed")
    return os.path.join(HERE, "libbmg.so")


if __name__ == "__main__":
    print(build(verbose=True))
