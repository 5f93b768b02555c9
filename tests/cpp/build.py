"""Build the C++ drop-in checks against the reference tree:

    python tests/cpp/build.py <reference checkout>

  tests/cpp/_build/drop_in   the reference's cg/gmres solver templates on the B200 backend tag
  tests/cpp/_build/stages    the reference's HeatProblem<CPU> beside the B200 heat problem, both driven
                             by the reference's unmodified stages and drivers

Both link residuum-solver_b200/librsd_cuda.so with an rpath relative to themselves, so they run
where the repository lies.  The stage check also compiles the reference's application sources it
links (expressions, solver instance, mesh generators, IO) from the checkout, with oracle/exprtk
standing in for the expression library the reference does not vendor.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build")


def _link(src, out, ref_root, extra_sources=(), extra_includes=()):
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ref_root, "include")]
    for inc in extra_includes:
        cmd += ["-I", inc]
    cmd += [src, *extra_sources, "-L", os.path.join(ROOT, "residuum-solver_b200"), "-lrsd_cuda",
            "-Wl,-rpath,$ORIGIN/../../../residuum-solver_b200", "-o", out]
    subprocess.run(cmd, check=True)


def build(ref_root):
    if not os.path.isdir(os.path.join(ref_root, "include")):
        return None
    os.makedirs(OUT, exist_ok=True)
    _link(os.path.join(HERE, "drop_in.cpp"), os.path.join(OUT, "drop_in"), ref_root)
    src = os.path.join(ref_root, "src")
    app = [os.path.join(src, p) for p in ("mesh/generator/BlockMesh2D.cpp", "mesh/generator/BlockMesh3D.cpp", "mesh/Mesh.cpp",
                                          "solver/SolverInstance.cpp", "utils/expression/ScalarExpression.cpp",
                                          "utils/expression/VectorExpression.cpp", "io/MeshIO.cpp")]
    app += sorted(glob.glob(os.path.join(src, "io", "visualization", "*.cpp")))
    _link(os.path.join(HERE, "stages.cpp"), os.path.join(OUT, "stages"), ref_root, app, [os.path.join(ROOT, "oracle", "exprtk")])
    return OUT


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: build.py <reference checkout>")
    print(build(sys.argv[1]))
