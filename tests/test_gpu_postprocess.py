"""GPU parity of the nodal field recovery (HeatProblem::computeNodalField: QuantityEvaluator with
SimpleAverageRecovery, heat flux and conductivity) against the C restatement, which
test_oracle_cpu.py pins bit for bit to the reference's own evaluator.

Tolerances: <= 1e-12 relative (max-abs error over max-abs value); exact linear fields to 1e-12.
"""
import numpy as np
import pytest

import oracle
from test_gpu_parity import distorted_mesh, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsd,order,nq,nel,kw", [
    (2, 1, 2, [7, 5], {}), (2, 2, 3, [4, 4], dict(k_expr="2 + T*T")), (2, 3, 4, [3, 2], {}),
    (3, 1, 2, [5, 4, 3], {}), (3, 2, 3, [3, 3, 2], dict(k_expr="1 + 0.5*T", dk_expr="0.5"))])
def test_nodal_fields_match_restatement(rsd, ctx, nsd, order, nq, nel, kw):
    m = distorted_mesh(nsd, order, nel, 5)
    ke = np.exp(0.3 * np.random.default_rng(2).standard_normal(m.nelem))
    bc = {0: "x", 1: "1"}
    o = oracle.Oracle(m, nq, bc=bc, src_expr="1", k_elem=ke, **kw)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, nsd, order, m.xyz, m.ien, m.rng), nq, src_expr="1", dirichlet=bc, k_elem=ke, **kw)
    U = np.cos(np.arange(o.n) * 0.37)
    Ud = ctx.to_device(U)
    assert relerr(h.nodal_field(Ud), o.nodal_field(U)) <= 1e-12
    assert relerr(h.nodal_field(Ud, "conductivity"), o.nodal_field(U, "conductivity")) <= 1e-12


def test_linear_temperature_gives_its_flux_everywhere(rsd, ctx):
    # T = 2x - 3y + z on every node (Dirichlet values included): Q = -k (2, -3, 1) at every node
    from test_gpu_parity import make_heat
    expr = "2*x - 3*y + z"
    h = make_heat(rsd, ctx, 3, 2, 3, [4, 3, 3], [0, 0, 0], [1, 2, 1.5], k_const=1.7,
                  dirichlet={t: expr for t in range(6)})
    t2a, a2t = h.dofmap()
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    X, _, _ = bm.block_mesh(3, [4, 3, 3], [0, 0, 0], [1, 2, 1.5], 2)
    X = X.reshape(-1, 3)[a2t]
    U = ctx.to_device(2 * X[:, 0] - 3 * X[:, 1] + X[:, 2])
    Q = h.nodal_field(U)
    assert np.max(np.abs(Q - (-1.7) * np.array([2.0, -3.0, 1.0]))) <= 1e-12 * 1.7 * 3
