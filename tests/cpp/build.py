"""Build tests/cpp/_build/drop_in: the reference's cg/gmres solver templates on the B200 backend tag.

    python tests/cpp/build.py [residuum include dir]

Needs the Residuum include/ tree (header-only parts) and residuum-solver_b200/librsd_cuda.so; the
binary links the library with an rpath relative to itself, so it runs where the repository lies.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "drop_in")


def build(ref_include):
    if not os.path.isdir(ref_include):
        return None
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", ref_include,
           os.path.join(HERE, "drop_in.cpp"), "-L", os.path.join(ROOT, "residuum-solver_b200"), "-lrsd_cuda",
           "-Wl,-rpath,$ORIGIN/../../../residuum-solver_b200", "-o", OUT]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/include"))
