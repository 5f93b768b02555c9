"""GPU parity of the matrix-free operator (operator type `fem`: FEMOperator products as element
passes, Jacobi from the element diagonal, FP64 CG) against the reference's own stages run with
OperatorType::FEM (golden fixtures from tests/golden/make_golden.py fem), and against this library's
CSR path on the same systems.

Tolerances: iteration counts equal to the reference's; solutions within 1e-12 relative (max-abs
error over max-abs value).  The k(T) case changes its operator while CG runs (the stage's state is
the solve's own iterate), so rounding differences grow over the iterations: 1e-9 there.
"""
import numpy as np
import pytest

from conftest import golden
from test_gpu_parity import make_heat, relerr

pytestmark = pytest.mark.gpu
REL = 1e-12


def fem_cfg(rsd, **kw):
    base = dict(type=rsd.CG, precond=rsd.JACOBI, tol=1e-10, max_iters=1000, operator_type=rsd.OP_FEM)
    base.update(kw)
    return rsd.SolverConfig.make(**base)


def test_steady_q1_hex_matches_reference(rsd, ctx):
    g = golden("fem_steady_q1_hex_6x5x4.npz")
    h = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], src_expr="x*y*z",
                  dirichlet={t: "x" for t in range(4)})
    U = ctx.array(h.n).zero()
    rep = h.steady(U, cfg=fem_cfg(rsd))
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert abs(rep["initialResidual"] - g["initialResidual"]) <= REL * g["initialResidual"]
    assert relerr(U.download(), g["U"]) <= REL
    assert rep["trueResidualRel"] <= 1e-9


def test_backward_euler_matches_reference(rsd, ctx):
    g = golden("fem_be_q1_hex_6x5x4.npz")
    h = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], dirichlet={t: "0" for t in range(6)})
    U, Up = ctx.to_device(g["U0"]), ctx.to_device(g["U0"])
    res, its = [], []
    for _ in range(5):
        rep = h.be_step(1e-2, U, Up, cfg=fem_cfg(rsd, tol=1e-8))
        assert rep["converged"]
        res.append(rep["residualNorm"])
        its.append(rep["iterations"])
    assert its == list(g["iterations"])
    assert relerr(U.download(), g["U"]) <= REL
    assert relerr(res, g["residual"]) <= 1e-9   # norms of residuals ~1e-8 of their parts: cancellation


def test_q2_elements_match_reference(rsd, ctx):
    g = golden("fem_steady_q2_quad_kelem.npz")
    h = make_heat(rsd, ctx, 2, 2, 3, [5, 3], [0, 0], [1, 1], src_expr="1", k_elem=g["k_elem"],
                  dirichlet={t: "(1-x)*(1-y)" for t in range(4)})
    U = ctx.array(h.n).zero()
    rep = h.steady(U, cfg=fem_cfg(rsd))
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert relerr(U.download(), g["U"]) <= REL
    g = golden("fem_steady_q2_hex_3x3x2.npz")
    h = make_heat(rsd, ctx, 3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1], src_expr="10", dirichlet={0: "0", 1: "1"})
    U = ctx.array(h.n).zero()
    rep = h.steady(U, cfg=fem_cfg(rsd))
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert relerr(U.download(), g["U"]) <= REL


def test_state_dependent_operator_matches_reference(rsd, ctx):
    g = golden("fem_steady_q2_hex_kT.npz")
    h = make_heat(rsd, ctx, 3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1], src_expr="10", k_expr="1 + 0.5*T",
                  dk_expr="0.5", dirichlet={0: "0", 1: "1"})
    U = ctx.array(h.n).zero()
    rep = h.steady(U, cfg=fem_cfg(rsd, tol=1e-12))
    assert bool(rep["converged"]) == bool(g["converged"])
    assert abs(rep["iterations"] - int(g["iterations"])) <= 1
    assert relerr(U.download(), g["U"]) <= 1e-9


@pytest.mark.parametrize("nsd,order,nq,nel", [(3, 1, 2, [9, 8, 7]), (2, 2, 3, [11, 9]), (3, 2, 3, [4, 3, 3])])
def test_matrix_free_solve_matches_csr_solve(rsd, ctx, nsd, order, nq, nel):
    # the same (Diffusion + c Mass) x = b through the assembled matrix and without it
    lo, hi = [0.0] * nsd, [1.0, 2.0, 1.5][:nsd]
    h = make_heat(rsd, ctx, nsd, order, nq, nel, lo, hi, src_expr="1", dirichlet={0: "0", 1: "1"})
    c = 37.0
    h.assemble_matrix(1.0, c)
    rng = np.random.default_rng(3)
    b = ctx.to_device(rng.standard_normal(h.n))
    x0 = 0.01 * rng.standard_normal(h.n)
    x1, x2 = ctx.to_device(x0), ctx.to_device(x0)
    cfg = rsd.SolverConfig.make(type=rsd.CG, precond=rsd.JACOBI, tol=1e-11, max_iters=5000)
    r1 = rsd.solve(ctx, h.K, b, x1, cfg)
    r2 = h.solve_fem(b, x2, c_mass=c, type=rsd.CG, precond=rsd.JACOBI, tol=1e-11, max_iters=5000)
    assert r1["converged"] and r2["converged"]
    assert abs(r1["iterations"] - r2["iterations"]) <= 1
    assert relerr(x2.download(), x1.download()) <= 1e-10
    assert r2["trueResidualRel"] <= 2e-11
    # the operator's product and diagonal against the assembled matrix
    v = ctx.to_device(rng.standard_normal(h.n))
    y1, y2 = ctx.array(h.n), ctx.array(h.n)
    h.K.spmv(v, y1)
    h.assemble_vector(4, y2, coef=c, operand=v)
    assert relerr(y2.download(), y1.download()) <= REL
    d1, d2 = ctx.array(h.n), ctx.array(h.n)
    h.K.diagonal(d1)
    h.diagonal(d2, c_diff=1.0, c_mass=c)
    assert relerr(d2.download(), d1.download()) <= REL


@pytest.mark.parametrize("nsd,order,nel", [(2, 1, [13, 9]), (2, 2, [7, 5]), (2, 3, [5, 4]), (3, 1, [7, 6, 5]),
                                           (3, 2, [4, 3, 3])])
def test_sum_factorized_product_matches_tables_and_matrix(rsd, ctx, monkeypatch, nsd, order, nel):
    # all-affine meshes with P+1 points per direction take the sum-factorized kernel; the table
    # kernel (RSD_SUMFAC=0) and the assembled matrix give the same product
    lo, hi = [0.0] * nsd, [1.0, 2.0, 1.5][:nsd]
    rng = np.random.default_rng(5)
    ke = np.exp(rng.standard_normal(int(np.prod(nel))))
    h = make_heat(rsd, ctx, nsd, order, order + 1, nel, lo, hi, k_elem=ke, rho=1.3, cp=0.7, k_const=2.5,
                  dirichlet={0: "0", 2: "1"})
    c = 11.0
    v = ctx.to_device(rng.standard_normal(h.n))
    y1, y2, y3 = ctx.array(h.n), ctx.array(h.n), ctx.array(h.n)
    h.assemble_matrix(1.0, c)
    h.K.spmv(v, y1)
    h.assemble_vector(4, y2, coef=c, operand=v)
    monkeypatch.setenv("RSD_SUMFAC", "0")
    h.assemble_vector(4, y3, coef=c, operand=v)
    assert relerr(y2.download(), y1.download()) <= REL
    assert relerr(y3.download(), y1.download()) <= REL
    if nsd == 3 and order == 2:
        # the 27-node kernel by lanes per node (shuffles) instead of lanes per grid line
        monkeypatch.setenv("RSD_SUMFAC", "1")
        monkeypatch.setenv("RSD_SUMFAC_PLANES", "0")
        h.assemble_vector(4, y3, coef=c, operand=v)
        assert relerr(y3.download(), y1.download()) <= REL
        monkeypatch.delenv("RSD_SUMFAC_PLANES")
    # the diffusion operator alone (coef 0)
    monkeypatch.delenv("RSD_SUMFAC")
    h.assemble_matrix(1.0, 0.0)
    h.K.spmv(v, y1)
    h.assemble_vector(4, y2, coef=0.0, operand=v)
    assert relerr(y2.download(), y1.download()) <= REL


def test_identity_preconditioner_and_limits(rsd, ctx):
    h = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], src_expr="1", dirichlet={t: "0" for t in range(6)})
    F = ctx.array(h.n)
    h.assemble_vector(0, F)
    x1, x2 = ctx.array(h.n).zero(), ctx.array(h.n).zero()
    h.assemble_matrix(1.0, 0.0)
    r1 = rsd.solve(ctx, h.K, F, x1, rsd.SolverConfig.make(type=rsd.CG, precond=rsd.IDENTITY, tol=1e-10))
    r2 = h.solve_fem(F, x2, type=rsd.CG, precond=rsd.IDENTITY, tol=1e-10)
    assert r1["iterations"] == r2["iterations"] and relerr(x2.download(), x1.download()) <= REL
    # max_iters reached: not converged, iterations = max_iters (cg/Solver.tpp:95-99)
    x2.zero()
    r = h.solve_fem(F, x2, type=rsd.CG, precond=rsd.JACOBI, tol=1e-30, max_iters=5)
    assert not r["converged"] and r["iterations"] == 5


def test_gmres_over_the_operator_matches_reference(rsd, ctx):
    g = golden("fem_steady_gmres7_q1_quad_16.npz")
    h = make_heat(rsd, ctx, 2, 1, 2, [16, 16], [0, 0], [1, 1], dirichlet={t: "(1-x)*(1-y)" for t in range(4)})
    U = ctx.array(h.n).zero()
    rep = h.steady(U, cfg=fem_cfg(rsd, type=rsd.GMRES, krylov_dim=7))
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert relerr(U.download(), g["U"]) <= REL
    # the same system through the assembled matrix
    U2 = ctx.array(h.n).zero()
    rep2 = h.steady(U2, type=rsd.GMRES, precond=rsd.JACOBI, tol=1e-10, max_iters=1000, krylov_dim=7)
    assert rep2["iterations"] == rep["iterations"] and relerr(U.download(), U2.download()) <= REL


def test_newton_with_the_jacobian_applied_matches_reference(rsd, ctx):
    # J = Diffusion + TangentDiffusion at the Newton state, never assembled; GMRES(30) + Jacobi from
    # its element diagonal, against the reference's Newton with operator type fem
    g = golden("fem_newton_q2_hex_3.npz")
    h = make_heat(rsd, ctx, 3, 2, 3, [3, 3, 3], [0, 0, 0], [1, 1, 1], src_expr="10", k_expr="1 + 0.5*T", dk_expr="0.5",
                  dirichlet={0: "0", 1: "1"})
    U = ctx.array(h.n).zero()
    cfg = rsd.SolverConfig.make(type=rsd.GMRES, precond=rsd.JACOBI, tol=1e-12, max_iters=1000, krylov_dim=30,
                                operator_type=rsd.OP_FEM)
    rep = h.newton(U, 1e-10, 1e-10, 50, cfg=cfg)
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert relerr(U.download(), g["U"]) <= 1e-11
    # the Jacobian product and diagonal against the assembled J = K + K_T
    rng = np.random.default_rng(9)
    Us = ctx.to_device(0.3 * rng.standard_normal(h.n))
    h.assemble_matrix(1.0, 0.0, 1.0, 0.0, U=Us)
    v = ctx.to_device(rng.standard_normal(h.n))
    y1 = ctx.array(h.n)
    h.K.spmv(v, y1)
    y2 = ctx.array(h.n)
    h.assemble_vector(10, y2, U=Us, operand=v)
    assert relerr(y2.download(), y1.download()) <= REL


def test_configurations_the_operator_does_not_take(rsd, ctx):
    h = make_heat(rsd, ctx, 2, 1, 2, [4, 4], [0, 0], [1, 1], src_expr="1", dirichlet={0: "0"})
    U, b = ctx.array(h.n).zero(), ctx.array(h.n).zero()
    for kw in (dict(precision=rsd.MIXED), dict(type=rsd.GMRES, krylov_dim=0)):
        with pytest.raises(rsd.RsdError, match="RSD_EINVAL"):
            h.steady(U, cfg=fem_cfg(rsd, **kw))
        with pytest.raises(rsd.RsdError, match="RSD_EINVAL"):
            h.solve_fem(b, U, **dict(dict(type=rsd.CG, tol=1e-8), **kw))
    # a matrix solve and the batched solver take the CSR operator only
    h.assemble_matrix(1.0, 0.0)
    with pytest.raises(rsd.RsdError, match="RSD_EINVAL"):
        rsd.solve(ctx, h.K, b, U, fem_cfg(rsd))
