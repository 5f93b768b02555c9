"""GPU parity of the flux (natural) boundary conditions: the reference's own known answers
(HeatEquationMinimal2D/3D natural-BC steps), and the stages with fluxes against the C restatement
(pinned to those answers in test_oracle_cpu.py) on the same seeded inputs.

Tolerances: known answers 1e-10 (the reference tests' own); vectors and solutions <= 1e-12 relative
(max-abs error over max-abs value); Newton solutions <= 1e-11.
"""
import numpy as np
import pytest

import oracle
from test_gpu_parity import distorted_mesh, make_heat, relerr

pytestmark = pytest.mark.gpu
REL = 1e-12


def test_known_answers_2d_and_3d(rsd, ctx):
    # HeatEquationMinimal2D.cpp:355-392: flux (0, x) on BOTTOM, then the lift
    h = make_heat(rsd, ctx, 2, 1, 2, [4, 4], [0, 0], [4, 4], src_expr="x*y", dirichlet={0: "x", 1: "x", 3: "x"},
                  flux={2: ("0", "x")})
    F = ctx.array(h.n)
    h.assemble_vector(0, F)
    h.apply_natural(F)
    h.lift(F, 1.0, 0.0)
    expect = [1 / 6 - 1, 1 / 3 - 2, 1 / 2 - 3 + 2, 1, 2, 3 + 4, 2, 4, 6 + 4, 3 + 1, 6 + 2, 9 + 17 / 3]
    assert np.max(np.abs(F.download() - expect)) <= 1e-10
    # HeatEquationMinimal3D.cpp:307-337: flux (0, 0, x) on BOTTOM and TOP
    h = make_heat(rsd, ctx, 3, 1, 2, [4, 4, 4], [0, 0, 0], [4, 4, 4], src_expr="x*y*z",
                  dirichlet={t: "x" for t in range(4)}, flux={4: ("0", "0", "x"), 5: ("0", "0", "x")})
    t2a, _ = h.dofmap()
    F = ctx.array(h.n)
    h.assemble_vector(0, F)
    h.apply_natural(F)
    F1 = F.download()
    Sz = [1 / 6, 1, 2, 3, 11 / 6]
    for i in range(1, 4):
        for j in range(1, 4):
            for k in range(5):
                e = i * j * Sz[k] + (-i if k == 0 else i if k == 4 else 0)
                assert abs(F1[t2a[i + 5 * j + 25 * k]] - e) <= 1e-10
    h.lift(F, 1.0, 0.0)
    F2 = F.download()
    for (i, j, k), e in (((1, 1, 0), -1 / 3), ((1, 1, 1), 2.0), ((1, 1, 4), 10 / 3), ((2, 2, 2), 8.0), ((3, 1, 1), 26 / 3)):
        assert abs(F2[t2a[i + 5 * j + 25 * k]] - e) <= 1e-10


@pytest.mark.parametrize("nsd,order,nq,nel", [(2, 1, 2, [7, 5]), (2, 2, 3, [5, 4]), (2, 3, 4, [3, 3]),
                                              (3, 1, 2, [5, 4, 3]), (3, 2, 3, [3, 3, 2])])
def test_flux_integrals_on_distorted_meshes(rsd, ctx, nsd, order, nq, nel):
    # position-dependent fluxes on several tags of a half-distorted mesh (curved faces' normals and
    # measures through cof(J)), against the restatement
    m = distorted_mesh(nsd, order, nel, 7)
    flux = {1: ("x*y", "1 + y") + (("z",) if nsd == 3 else ()),
            2: ("sin(x)", "x*x") + (("0.5",) if nsd == 3 else ()),
            3: ("0", "2") + (("x - z",) if nsd == 3 else ())}
    bc = {0: "x"}
    o = oracle.Oracle(m, nq, bc=bc, src_expr="1", flux=flux)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, nsd, order, m.xyz, m.ien, m.rng), nq, src_expr="1", dirichlet=bc, flux=flux)
    F = ctx.array(h.n).zero()
    h.apply_natural(F)
    assert relerr(F.download(), o.natural(np.zeros(o.n))) <= REL
    # clearing a tag removes its terms only
    h.set_flux(2, None)
    F.zero()
    h.apply_natural(F)
    o2 = oracle.Oracle(m, nq, bc=bc, src_expr="1", flux={1: flux[1], 3: flux[3]})
    assert relerr(F.download(), o2.natural(np.zeros(o2.n))) <= REL


def test_stages_with_flux_match_restatement(rsd, ctx):
    # steady (CSR and matrix-free), Backward Euler with a time-dependent flux, and Newton with k(T)
    bm = oracle.BlockMesh(3, [6, 5, 4], [0, 0, 0], [1, 1, 1], 1)
    flux = {1: ("1", "0", "0"), 4: ("0", "0", "-2*x")}
    bc = {0: "0", 2: "0.5"}
    o = oracle.Oracle(bm, 2, bc=bc, src_expr="1", flux=flux)
    h = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], src_expr="1", dirichlet=bc, flux=flux)
    Uo, ro = o.steady(tol=1e-10)
    U = ctx.array(h.n).zero()
    rep = h.steady(U, type=rsd.CG, precond=rsd.JACOBI, tol=1e-10)
    assert rep["iterations"] == ro["iterations"] and relerr(U.download(), Uo) <= REL
    U.zero()
    rep = h.steady(U, type=rsd.CG, precond=rsd.JACOBI, tol=1e-10, operator_type=rsd.OP_FEM)
    assert rep["iterations"] == ro["iterations"] and relerr(U.download(), Uo) <= REL
    # Backward Euler: the flux is evaluated at each step's time
    flux_t = {1: ("t*x", "0", "0"), 5: ("0", "0", "1 + t")}
    o = oracle.Oracle(bm, 2, bc=bc, src_expr="1", flux=flux_t)
    h = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], src_expr="1", dirichlet=bc, flux=flux_t)
    U0 = np.cos(np.arange(o.n) * 0.3)
    Uo, reso, _, _ = o.backward_euler(0.05, 4, U0, tol=1e-10)
    U, Up = ctx.to_device(U0), ctx.to_device(U0)
    res = [h.be_step(0.05, U, Up, type=rsd.CG, precond=rsd.JACOBI, tol=1e-10)["residualNorm"] for _ in range(4)]
    assert relerr(U.download(), Uo) <= REL
    assert relerr(res, reso) <= 1e-9
    # Newton with k(T) and a flux on the far side
    q2 = oracle.BlockMesh(3, [3, 3, 2], [0, 0, 0], [1, 1, 1], 2)
    kw = dict(src_expr="10", k_expr="1 + 0.5*T", dk_expr="0.5")
    fl = {1: ("0.3 + y", "0", "0")}
    o = oracle.Oracle(q2, 3, bc={0: "0"}, flux=fl, **kw)
    Uo, ro = o.newton(1e-10, 1e-10, 50, solver=1, precond=1, tol=1e-12, krylov=30)
    h = make_heat(rsd, ctx, 3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1], dirichlet={0: "0"}, flux=fl, **kw)
    U = ctx.array(h.n).zero()
    cfg = rsd.SolverConfig.make(type=rsd.GMRES, precond=rsd.JACOBI, tol=1e-12, max_iters=1000, krylov_dim=30)
    rep = h.newton(U, 1e-10, 1e-10, 50, cfg=cfg)
    assert rep["converged"] and rep["iterations"] == ro["iterations"]
    assert relerr(U.download(), Uo) <= 1e-11


def test_flux_arguments(rsd, ctx):
    h = make_heat(rsd, ctx, 2, 1, 2, [3, 3], [0, 0], [1, 1], dirichlet={0: "0"})
    with pytest.raises(rsd.RsdError, match="RSD_EINVAL"):
        h.set_flux(-1, ("1", "0"))         # boundary tags are >= 0
    h.set_flux(9, ("1", "0"))              # any tag may carry a flux; no face has tag 9 here
    F9 = ctx.array(h.n).zero()
    h.apply_natural(F9)
    assert not np.any(F9.download())
    h.set_flux(9, None)
    with pytest.raises(rsd.RsdError, match="RSD_EPARSE"):
        h.set_flux(1, ("1 +", "0"))
    h.set_flux(1, ("1", "0"))
    F = ctx.array(h.n).zero()
    h.apply_natural(F)
    assert abs(F.download().sum() - 1.0) <= 1e-12 * h.n   # unit flux through the x = 1 edge of length 1
