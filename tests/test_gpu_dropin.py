"""The reference's own cg::Solver and gmres::Solver templates, unmodified, run on device data through
the C++20 backend tag of include/rsd_residuum.hpp (tests/cpp/drop_in.cpp), against the same
templates on the reference's CPU tag."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp", "_build", "drop_in")


def test_reference_solvers_on_the_b200_tag():
    if not os.path.exists(BIN):
        pytest.skip("tests/cpp/_build/drop_in not built (needs the reference headers at build time)")
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    d = json.loads(out.stdout)
    for name in ("cg_jacobi", "gmres20_jacobi"):
        c, g = d[name]["cpu"], d[name]["b200"]
        assert c["converged"] and g["converged"], d[name]
        assert abs(c["iterations"] - g["iterations"]) <= 1, d[name]
        assert abs(g["res0"] - c["res0"]) <= 1e-12 * c["res0"]
        assert g["res"] / g["res0"] < 1e-10
        assert d[name]["x_rel_diff"] <= 1e-8, d[name]
