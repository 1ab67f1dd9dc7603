"""Build the in-tree CUDA library (nvcc, sm_100a) with the committed Makefile.

``python -m frforge_b200.build`` compiles ``libfrforge_cuda.so`` next to this
file; nvcc cross-compiles, so no GPU is needed.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, quiet: bool = True) -> str:
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return os.path.join(HERE, "libfrforge_cuda.so")


if __name__ == "__main__":
    print(build(quiet="-v" not in sys.argv))
