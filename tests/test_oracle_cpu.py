"""CPU tests of the checkers: the C restatement against the reference's own known-answer tests,
against the golden fixtures, and (where oracle/_ref was built) against the reference templates."""
import numpy as np
import pytest

import oracle
from conftest import golden, load_package

TOL = 1e-10  # the reference tests' own tolerance for these known answers


@pytest.fixture(scope="module")
def mini2d():
    m = oracle.BlockMesh(2, [4, 4], [0, 0], [4, 4], 1)
    return oracle.Oracle(m, 2, src_expr="x*y", bc={0: "x", 1: "x", 3: "x"})


@pytest.fixture(scope="module")
def mini3d():
    m = oracle.BlockMesh(3, [4, 4, 4], [0, 0, 0], [4, 4, 4], 1)
    return oracle.Oracle(m, 2, src_expr="x*y*z", bc={0: "x", 1: "x", 2: "x", 3: "x"})


def csr_dense(rp, col, val, n):
    A = np.zeros((n, n))
    for i in range(n):
        A[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    return A


def test_dofmap_2d_known_answers(mini2d):
    # tests/integration/fem/heateq/cpu/HeatEquationMinimal2D.cpp:157-208
    t2a, a2t, ctag = mini2d.dofmap()
    assert mini2d.mesh.nnodes == 25 and mini2d.n == 12
    for i in list(range(0, 21, 5)) + list(range(4, 25, 5)) + [21, 22]:
        assert t2a[i] == -1
    expect = {1: 0, 2: 1, 3: 2, 6: 3, 7: 4, 8: 5, 11: 6, 12: 7, 13: 8, 16: 9, 17: 10, 18: 11}
    for topo, alg in expect.items():
        assert t2a[topo] == alg and a2t[alg] == topo
    assert ctag[10] == 0 and ctag[15] == 0 and ctag[21] == 3 and ctag[9] == 1


def test_matrix_2d_known_answers(mini2d):
    # HeatEquationMinimal2D.cpp:240-271
    rp, col = mini2d.pattern()
    K = csr_dense(rp, col, mini2d.assemble_matrix(), 12)
    assert np.allclose(np.diag(K)[:3], 4 / 3, atol=TOL) and np.allclose(np.diag(K)[3:], 8 / 3, atol=TOL)
    for i in range(2):
        assert abs(K[i, i + 1] + 1 / 6) < TOL and abs(K[i + 1, i] + 1 / 6) < TOL
    for i in [3, 6, 7, 9, 10]:
        assert abs(K[i, i + 1] + 1 / 3) < TOL
    for i in range(9):
        assert abs(K[i, i + 3] + 1 / 3) < TOL and abs(K[i + 3, i] + 1 / 3) < TOL


def test_vectors_2d_known_answers(mini2d):
    # O = K.1 (HeatEquationMinimal2D.cpp:305-326); F and the essential increments (:353-398)
    O = mini2d.assemble_vector(4, 0.0, operand=np.ones(12))
    expect = [0.5, 0.0, 0.5, 1.0, 0.0, 1.0, 1.0, 0.0, 1.0, 5 / 3, 1.0, 5 / 3]
    assert np.allclose(O, expect, atol=TOL)
    F = mini2d.assemble_vector(0)
    assert np.allclose(F, [1 / 6, 1 / 3, 1 / 2, 1, 2, 3, 2, 4, 6, 3, 6, 9], atol=TOL)
    inc = mini2d.lift(F) - F
    assert np.allclose(inc, [0, 0, 2, 0, 0, 4, 0, 0, 4, 1, 2, 17 / 3], atol=TOL)


def test_3d_known_answers(mini3d):
    # tests/integration/fem/heateq/cpu/HeatEquationMinimal3D.cpp:168-329
    t2a, _, ctag = mini3d.dofmap()
    nid = lambda i, j, k: 25 * k + 5 * j + i
    assert mini3d.n == 45
    assert t2a[nid(2, 2, 2)] >= 0 and t2a[nid(1, 1, 0)] >= 0 and t2a[nid(0, 2, 2)] == -1
    assert ctag[nid(0, 2, 2)] == 0 and ctag[nid(4, 2, 2)] == 1 and ctag[nid(2, 0, 2)] == 2 and ctag[nid(2, 4, 2)] == 3
    rp, col = mini3d.pattern()
    K = csr_dense(rp, col, mini3d.assemble_matrix(), 45)
    for i in range(1, 4):
        for j in range(1, 4):
            for k in range(5):
                a = t2a[nid(i, j, k)]
                assert abs(K[a, a] - (4 / 3 if k in (0, 4) else 8 / 3)) < TOL
    c = t2a[nid(2, 2, 2)]
    assert abs(K[c, t2a[nid(2, 2, 1)]]) < TOL
    assert abs(K[c, t2a[nid(1, 1, 2)]] + 1 / 6) < TOL
    assert abs(K[c, t2a[nid(1, 1, 1)]] + 1 / 12) < TOL
    O = mini3d.assemble_vector(4, 0.0, operand=np.ones(45))
    for k in range(5):
        assert abs(O[t2a[nid(2, 2, k)]]) < TOL
        assert abs(O[t2a[nid(1, 1, k)]] - (5 / 6 if k in (0, 4) else 5 / 3)) < TOL
    F = mini3d.assemble_vector(0)
    Sz = [1 / 6, 1, 2, 3, 11 / 6]
    for i in range(1, 4):
        for j in range(1, 4):
            for k in range(5):
                assert abs(F[t2a[nid(i, j, k)]] - i * j * Sz[k]) < TOL
    # the essential increments at the spot-checked nodes: final value minus (source + flux) value
    inc = mini3d.lift(F) - F
    flux = {nid(1, 1, 0): -1.0, nid(1, 1, 4): 1.0}
    spots = {nid(1, 1, 0): -1 / 3, nid(1, 1, 1): 2.0, nid(1, 1, 4): 10 / 3, nid(2, 2, 2): 8.0, nid(3, 1, 1): 26 / 3}
    for node, final in spots.items():
        before = F[t2a[node]] + flux.get(node, 0.0)
        assert abs(inc[t2a[node]] - (final - before)) < TOL


def test_cg_gmres_jacobi_known_answers():
    # tests/unit/linalg/solver/iterative/cg/Solver.cpp:12-68: [[4,1],[1,3]] x = [1,2] -> (1/11, 7/11)
    x, rep = oracle.csr_solve([0, 2, 4], [0, 1, 0, 1], [4, 1, 1, 3], [1, 2], tol=1e-12)
    assert rep["converged"] and np.allclose(x, [1 / 11, 7 / 11], atol=1e-10)
    # gmres/Solver.cpp:12-172: nonsymmetric [[2,1],[3,4]] x = [1,3] -> (1/5, 3/5)
    A = np.array([[2.0, 1.0], [3.0, 4.0]])
    b = np.array([1.0, 3.0])
    x, rep = oracle.csr_solve([0, 2, 4], [0, 1, 0, 1], A.ravel(), b, solver=1, krylov=2, tol=1e-12)
    assert rep["converged"] and np.allclose(A @ x, b, atol=1e-10)
    # restart with m = 1 still converges
    x, rep = oracle.csr_solve([0, 2, 4], [0, 1, 0, 1], A.ravel(), b, solver=1, krylov=1, tol=1e-10, maxit=200)
    assert rep["converged"] and np.allclose(A @ x, b, atol=1e-8)
    # Jacobi: a zero diagonal falls back to 1 (Jacobi.hpp:33) and the solve still runs
    x, rep = oracle.csr_solve([0, 1, 2], [0, 1], [1e-320, 2.0], [0.0, 4.0], tol=1e-12, maxit=5)
    assert np.isfinite(x).all()


def test_expression_language():
    assert oracle.expr_eval("(1-x)*(1-y)", x=0.25, y=0.5) == (1 - 0.25) * (1 - 0.5)
    assert abs(oracle.expr_eval("1 + 0.5*T", T=2.0) - 2.0) < 1e-15
    assert abs(oracle.expr_eval("-2^2") + 4.0) < 1e-15
    assert abs(oracle.expr_eval("sin(pi*x)", x=0.5) - 1.0) < 1e-15
    with pytest.raises(ValueError):
        oracle.expr_eval("not an expression (")


@pytest.mark.parametrize("name,nsd,order,nq,nel,lo,hi,bc,src,kw", [
    ("q1_quad_4x4.npz", 2, 1, 2, [4, 4], [0, 0], [4, 4], {0: "x", 1: "x", 3: "x"}, "x*y", {}),
    ("q1_hex_4x4x4.npz", 3, 1, 2, [4, 4, 4], [0, 0, 0], [4, 4, 4], {t: "x" for t in range(4)}, "x*y*z", {}),
    ("q2_hex_3x3x2.npz", 3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1], {0: "0", 1: "1"}, "10",
     {"k_expr": "1 + 0.5*T", "dk_expr": "0.5"}),
    ("q2_quad_kelem.npz", 2, 2, 3, [5, 3], [0, 0], [1, 1], {t: "(1-x)*(1-y)" for t in range(4)}, "1", {"kelem": True}),
])
def test_restatement_matches_golden(name, nsd, order, nq, nel, lo, hi, bc, src, kw):
    g = golden(name)
    m = oracle.BlockMesh(nsd, nel, lo, hi, order)
    o = oracle.Oracle(m, nq, k_expr=kw.get("k_expr"), dk_expr=kw.get("dk_expr"),
                      k_elem=g.get("k_elem") if kw.get("kelem") else None, src_expr=src, bc=bc)
    t2a, a2t, _ = o.dofmap()
    rp, col = o.pattern()
    assert (t2a == g["t2a"]).all() and (a2t == g["a2t"]).all()
    assert (rp == g["row_ptr"]).all() and (col == g["col"]).all()
    U, Ud = g["U"], g["Udot"]
    # the restatement follows the reference's accumulation order: bit-identical
    assert (o.assemble_matrix(U=U) == g["K"]).all()
    assert (o.assemble_matrix(1, 7.5, U=U) == g["K_cM"]).all()
    assert (o.assemble_matrix(1, 0, 1, 0, U=U) == g["K_KT"]).all()
    F = o.assemble_vector(0)
    assert (F == g["F"]).all()
    assert (o.lift(F) - F == g["lift"]).all()
    assert (o.lift(F, 1.0, 7.5) - F == g["lift_cM"]).all()
    assert (o.assemble_vector(4, 0.0, operand=np.ones(o.n)) == g["O_ones"]).all()
    assert (o.assemble_vector(4, 2.5, operand=Ud) == g["O_cM"]).all()
    assert (o.assemble_vector(1, U=U) == g["R_diff"]).all()
    assert (o.assemble_vector(2, U=U) == g["M_U"]).all()
    assert (o.assemble_vector(3, Udot=Ud) == g["M_Udot"]).all()
    assert (o.diagonal(1.0, 7.5, U=U) == g["diag"]).all()


def test_restatement_stages_match_golden():
    g = golden("steady_q1_quad_16.npz")
    m = oracle.BlockMesh(2, [16, 16], [0, 0], [1, 1], 1)
    o = oracle.Oracle(m, 2, bc={t: "(1-x)*(1-y)" for t in range(4)})
    U, rep = o.steady(0, 1, 1e-10, 1000)
    assert rep["iterations"] == g["iterations"] and (U == g["U"]).all()
    g = golden("steady_gmres7_q1_quad_16.npz")
    U, rep = o.steady(1, 1, 1e-10, 1000, 7)
    assert rep["iterations"] == g["iterations"] and (U == g["U"]).all()
    g = golden("be_q1_hex_6x5x4.npz")
    m = oracle.BlockMesh(3, [6, 5, 4], [0, 0, 0], [1, 1, 1], 1)
    o = oracle.Oracle(m, 2, bc={t: "0" for t in range(6)})
    U, res, its, rc = o.backward_euler(1e-2, 5, g["U0"], tol=1e-8)
    assert rc == 0 and (U == g["U"]).all() and (res == g["residual"]).all()
    g = golden("newton_q2_hex_3.npz")
    m = oracle.BlockMesh(3, [3, 3, 3], [0, 0, 0], [1, 1, 1], 2)
    o = oracle.Oracle(m, 3, k_expr="1 + 0.5*T", dk_expr="0.5", src_expr="10", bc={0: "0", 1: "1"})
    U, rep = o.newton()
    assert rep["iterations"] == g["iterations"] and (U == g["U"]).all()


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built (reference tree absent)")
def test_restatement_matches_reference_bcs_time_dependent():
    # BE with a time-dependent Dirichlet value: the reference evaluates it at t and at t - dt
    m = oracle.BlockMesh(2, [6, 4], [0, 0], [1, 1], 1)
    o = oracle.Oracle(m, 2, bc={0: "0", 1: "0"}, src_expr="1")
    r = oracle.Reference(2, 1, 2, [6, 4], [0, 0], [1, 1], [0, 1], bc_kind=0, src_kind=0, src_c=1.0)
    U0 = np.linspace(0, 1, o.n)
    Uo, reso, _, _ = o.backward_euler(0.05, 4, U0, tol=1e-10)
    Ur, resr, _ = r.backward_euler(0.05, 4, U0, tol=1e-10)
    assert (Uo == Ur).all() and (reso == resr).all()


def test_restatement_matrix_free_operator_matches_golden():
    # the reference stages with operator type "fem" (FEMOperator): steady, Backward Euler and a
    # state-dependent k(T) whose operator follows the CG iterate; the restatement is bit-exact
    m = oracle.BlockMesh(3, [6, 5, 4], [0, 0, 0], [1, 1, 1], 1)
    o = oracle.Oracle(m, 2, bc={t: "x" for t in range(4)}, src_expr="x*y*z")
    o.set_operator("fem")
    U, rep = o.steady(tol=1e-10)
    g = golden("fem_steady_q1_hex_6x5x4.npz")
    assert rep["iterations"] == g["iterations"] and (U == g["U"]).all()
    o = oracle.Oracle(m, 2, bc={t: "0" for t in range(6)})
    o.set_operator("fem")
    g = golden("fem_be_q1_hex_6x5x4.npz")
    U, res, its, rc = o.backward_euler(1e-2, 5, g["U0"], tol=1e-8)
    assert rc == 0 and (its == g["iterations"]).all() and (U == g["U"]).all() and (res == g["residual"]).all()
    g = golden("fem_steady_q2_quad_kelem.npz")
    m2 = oracle.BlockMesh(2, [5, 3], [0, 0], [1, 1], 2)
    o = oracle.Oracle(m2, 3, bc={t: "(1-x)*(1-y)" for t in range(4)}, src_expr="1", k_elem=g["k_elem"])
    o.set_operator("fem")
    U, rep = o.steady(tol=1e-10)
    assert rep["iterations"] == g["iterations"] and (U == g["U"]).all()
    m3 = oracle.BlockMesh(3, [3, 3, 2], [0, 0, 0], [1, 1, 1], 2)
    for name, kw, tol in (("fem_steady_q2_hex_3x3x2.npz", {}, 1e-10),
                          ("fem_steady_q2_hex_kT.npz", dict(k_expr="1 + 0.5*T", dk_expr="0.5"), 1e-12)):
        g = golden(name)
        o = oracle.Oracle(m3, 3, bc={0: "0", 1: "1"}, src_expr="10", **kw)
        o.set_operator("fem")
        U, rep = o.steady(tol=tol)
        assert rep["iterations"] == g["iterations"] and (U == g["U"]).all()
    # matrix-free and assembled operators solve the same constant-k system
    o = oracle.Oracle(m, 2, bc={0: "0", 1: "1"}, src_expr="1")
    Uc, rc_ = o.steady(tol=1e-12)
    o.set_operator("fem")
    Uf, rf = o.steady(tol=1e-12)
    assert abs(rc_["iterations"] - rf["iterations"]) <= 1
    assert np.max(np.abs(Uf - Uc)) <= 1e-12 * np.max(np.abs(Uc))


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built (reference tree absent)")
def test_matrix_free_fixtures_reproduce_from_reference():
    r = oracle.Reference(3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0)
    r.set_operator("fem")
    g = golden("fem_be_q1_hex_6x5x4.npz")
    U, res, rc = r.backward_euler(1e-2, 5, g["U0"], tol=1e-8)
    assert rc == 0 and (U == g["U"]).all() and (res == g["residual"]).all()


def test_natural_bcs_known_answers():
    # tests/integration/fem/heateq/cpu/HeatEquationMinimal2D.cpp:96-112, 355-392: flux h = (0, x) on
    # BOTTOM adds -1, -2, -3 to the three free bottom nodes, then the lift
    m = oracle.BlockMesh(2, [4, 4], [0, 0], [4, 4], 1)
    o = oracle.Oracle(m, 2, src_expr="x*y", bc={0: "x", 1: "x", 3: "x"}, flux={2: ("0", "x")})
    F = o.lift(o.natural(o.assemble_vector(0)), 1.0, 0.0)
    expect = [1 / 6 - 1, 1 / 3 - 2, 1 / 2 - 3 + 2, 1, 2, 3 + 4, 2, 4, 6 + 4, 3 + 1, 6 + 2, 9 + 17 / 3]
    assert np.max(np.abs(F - expect)) <= TOL
    # HeatEquationMinimal3D.cpp:288-337: flux (0, 0, x) on BOTTOM/TOP adds -i / +i on the k = 0 / 4 layers
    m = oracle.BlockMesh(3, [4, 4, 4], [0, 0, 0], [4, 4, 4], 1)
    o = oracle.Oracle(m, 2, src_expr="x*y*z", bc={t: "x" for t in range(4)}, flux={4: ("0", "0", "x"), 5: ("0", "0", "x")})
    t2a, _, _ = o.dofmap()
    F0 = o.assemble_vector(0)
    F1 = o.natural(F0)
    Sz = [1 / 6, 1, 2, 3, 11 / 6]
    for i in range(1, 4):
        for j in range(1, 4):
            for k in range(5):
                a = t2a[i + 5 * j + 25 * k]
                e = i * j * Sz[k] + (-i if k == 0 else i if k == 4 else 0)
                assert abs(F1[a] - e) <= TOL
    F2 = o.lift(F1, 1.0, 0.0)
    node = lambda i, j, k: t2a[i + 5 * j + 25 * k]
    for (i, j, k), e in (((1, 1, 0), -1 / 3), ((1, 1, 1), 2.0), ((1, 1, 4), 10 / 3), ((2, 2, 2), 8.0), ((3, 1, 1), 26 / 3)):
        assert abs(F2[node(i, j, k)] - e) <= TOL


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built (reference tree absent)")
def test_nodal_field_recovery_matches_reference():
    # QuantityEvaluator::evaluateNodalField with SimpleAverageRecovery (heat flux, conductivity):
    # the restatement is bit-exact with the reference's own evaluator
    for nsd, order, nq, nel, kw, rk in [(2, 1, 2, [5, 4], {}, {}), (3, 1, 2, [4, 3, 3], {}, {}),
                                        (3, 2, 3, [3, 2, 2], dict(k_expr="1 + 0.5*T"), dict(k_a=1.0, k_b=0.5))]:
        r = oracle.Reference(nsd, order, nq, nel, [0] * nsd, [1] * nsd, [0, 1], bc_kind=0, bc_val={0: 0.0, 1: 1.0},
                             src_kind=0, src_c=1.0, **rk)
        m = oracle.BlockMesh(nsd, nel, [0] * nsd, [1] * nsd, order)
        o = oracle.Oracle(m, nq, bc={0: "0", 1: "1"}, src_expr="1", **kw)
        U = np.sin(np.arange(o.n) * 0.7)
        assert (r.nodal_field(U) == o.nodal_field(U)).all()
        assert (r.nodal_field(U, "conductivity") == o.nodal_field(U, "conductivity")).all()


def test_blockmesh_generator_matches_restatement():
    rsd = load_package()
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    for nsd, nel, order in [(2, [5, 3], 1), (2, [4, 2], 2), (3, [3, 4, 2], 1), (3, [2, 2, 3], 2)]:
        m = oracle.BlockMesh(nsd, nel, [0.0] * nsd, [1.0, 2.0, 3.0][:nsd], order)
        xyz, ien, rng = bm.block_mesh(nsd, nel, [0.0] * nsd, [1.0, 2.0, 3.0][:nsd], order)
        assert (xyz == m.xyz).all() and (ien == m.ien).all() and (rng == m.rng).all()
    assert rsd.LIB_PATH.endswith("librsd_cuda.so")
