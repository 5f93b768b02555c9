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


STAGES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp", "_build", "stages")


def test_reference_stages_on_the_b200_heat_problem():
    """The reference's HeatProblem<CPU> and the B200 heat problem (include/rsd_residuum_heat.hpp) built
    from the same HeatConfig and driven by the same unmodified SteadyStage / BackwardEulerStage /
    NewtonRunner / Steady and Transient drivers reach the same states: steady CSR (device CG and the
    reference's cg::Solver on the tag), Backward Euler with the assembled and the matrix-free
    operator, Q2 Newton with both operators, a Backward-Euler Newton with an anisotropic k(T), cp(T)
    (TangentMass), a renumbered tag, a time-dependent Dirichlet value and a flux boundary, and a
    constant anisotropic Q2 quad problem."""
    if not os.path.exists(STAGES):
        pytest.skip("tests/cpp/_build/stages not built (needs the reference tree at build time)")
    out = subprocess.run([STAGES], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    d = json.loads(out.stdout)
    assert len(d) == 8, d
    for name, r in d.items():
        assert r["cpu_ok"] and r["b200_ok"], (name, r)
        assert r["n"] == r["n_b200"], (name, r)
        assert r["max_abs"] > 0.0, (name, r)
        # FP64 on both sides, the same iterations: the states agree to rounding
        assert r["rel_diff"] <= 1e-12, (name, r)
