"""GPU parity: the CUDA path through the C ABI against the golden fixtures (the reference
templates' own output) and the C restatement, on the same seeded inputs.

Tolerances: integer work (DOF map, CSR pattern) is bit-exact; FP64 values and solutions agree to
<= 1e-12 relative (max-abs error over max-abs value); FP32 work states its own bound in each test.
"""
from importlib import import_module

import numpy as np
import pytest

import oracle
from conftest import golden

pytestmark = pytest.mark.gpu
REL = 1e-12


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def bm():
    return import_module("residuum_solver_b200.blockmesh")


def make_heat(rsd, ctx, nsd, order, nq, nel, lo, hi, **kw):
    xyz, ien, rng = bm().block_mesh(nsd, nel, lo, hi, order)
    mesh = rsd.Mesh(ctx, nsd, order, xyz, ien, rng)
    return rsd.Heat(ctx, mesh, nq, **kw)


CASES = [
    ("q1_quad_4x4.npz", 2, 1, 2, [4, 4], [0, 0], [4, 4], dict(src_expr="x*y", dirichlet={0: "x", 1: "x", 3: "x"})),
    ("q1_hex_4x4x4.npz", 3, 1, 2, [4, 4, 4], [0, 0, 0], [4, 4, 4], dict(src_expr="x*y*z", dirichlet={t: "x" for t in range(4)})),
    ("q2_hex_3x3x2.npz", 3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1],
     dict(src_expr="10", k_expr="1 + 0.5*T", dk_expr="0.5", dirichlet={0: "0", 1: "1"})),
    ("q2_quad_kelem.npz", 2, 2, 3, [5, 3], [0, 0], [1, 1], dict(src_expr="1", dirichlet={t: "(1-x)*(1-y)" for t in range(4)})),
]


@pytest.mark.parametrize("name,nsd,order,nq,nel,lo,hi,kw", CASES)
def test_element_loops_match_reference(rsd, ctx, name, nsd, order, nq, nel, lo, hi, kw):
    g = golden(name)
    if "k_elem" in g:
        kw = dict(kw, k_elem=g["k_elem"])
    h = make_heat(rsd, ctx, nsd, order, nq, nel, lo, hi, **kw)
    t2a, a2t = h.dofmap()
    assert (t2a == g["t2a"]).all() and (a2t == g["a2t"]).all()            # bit-exact DOF map
    rp, col = h.K.pattern()
    assert (rp == g["row_ptr"]).all() and (col == g["col"]).all()         # bit-exact pattern
    n = h.n
    U, Ud = ctx.to_device(g["U"]), ctx.to_device(g["Udot"])
    h.assemble_matrix(U=U)
    assert relerr(h.K.values(), g["K"]) <= REL
    h.assemble_matrix(1.0, 7.5, U=U)
    assert relerr(h.K.values(), g["K_cM"]) <= REL
    h.assemble_matrix(1.0, 0.0, 1.0, 0.0, U=U)
    assert relerr(h.K.values(), g["K_KT"]) <= REL
    out = ctx.array(n)
    h.assemble_vector(0, out)
    F = out.download()
    assert relerr(F, g["F"]) <= REL
    Fd = ctx.to_device(g["F"])
    h.lift(Fd)
    assert relerr(Fd.download() - g["F"], g["lift"]) <= REL
    Fd = ctx.to_device(g["F"])
    h.lift(Fd, 1.0, 7.5)
    assert relerr(Fd.download() - g["F"], g["lift_cM"]) <= REL
    ones = ctx.to_device(np.ones(n))
    h.assemble_vector(4, out, coef=0.0, operand=ones)
    assert relerr(out.download(), g["O_ones"]) <= REL
    h.assemble_vector(4, out, coef=2.5, operand=Ud)
    assert relerr(out.download(), g["O_cM"]) <= REL
    h.assemble_vector(1, out, U=U)
    assert relerr(out.download(), g["R_diff"]) <= REL
    h.assemble_vector(2, out, U=U)
    assert relerr(out.download(), g["M_U"]) <= REL
    h.assemble_vector(3, out, Udot=Ud)
    assert relerr(out.download(), g["M_Udot"]) <= REL
    h.diagonal(out, 1.0, 7.5, U=U)
    assert relerr(out.download(), g["diag"]) <= REL


def distorted_mesh(nsd, order, nel, seed):
    # block mesh with the nodes of the left half moved at random (the restatement's own copy is
    # moved too): elements there are not affine, those on the right stay affine, so one launch
    # takes both the quadrature path and the reference-integral path
    m = oracle.BlockMesh(nsd, nel, [0] * nsd, [1] * nsd, order)
    X = np.ctypeslib.as_array(m._m.xyz, shape=(m.nnodes, nsd))
    rng = np.random.default_rng(seed)
    move = ((X > 1e-9) & (X < 1 - 1e-9)).all(1) & (X[:, 0] < 0.45)
    X[move] += (0.2 / (order * max(nel))) * rng.uniform(-1.0, 1.0, (int(move.sum()), nsd))
    m.xyz = X.reshape(-1).copy()
    return m


@pytest.mark.parametrize("nsd,order,nq,nel", [(3, 1, 2, [6, 5, 4]), (2, 2, 3, [5, 3]), (3, 2, 3, [3, 2, 2])])
def test_distorted_and_affine_elements_match_reference(rsd, ctx, nsd, order, nq, nel):
    m = distorted_mesh(nsd, order, nel, 11)
    bc = {0: "x", 1: "0"}
    o = oracle.Oracle(m, nq, rho=1.5, cp=2.0, bc=bc)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, nsd, order, m.xyz, m.ien, m.rng), nq, rho=1.5, cp=2.0, dirichlet=bc)
    n = h.n
    rng = np.random.default_rng(3)
    Uh, Udh = rng.standard_normal(n), rng.standard_normal(n)
    U, Ud = ctx.to_device(Uh), ctx.to_device(Udh)
    h.assemble_matrix(1.0, 7.5)
    assert relerr(h.K.values(), o.assemble_matrix(1.0, 7.5)) <= REL
    out = ctx.array(n)
    h.assemble_vector(1, out, U=U)
    assert relerr(out.download(), o.assemble_vector(1, U=Uh)) <= REL
    h.assemble_vector(2, out, U=U)
    assert relerr(out.download(), o.assemble_vector(2, U=Uh)) <= REL
    h.assemble_vector(3, out, Udot=Ud)
    assert relerr(out.download(), o.assemble_vector(3, Udot=Udh)) <= REL
    h.assemble_vector(4, out, coef=2.5, operand=Ud)
    assert relerr(out.download(), o.assemble_vector(4, coef=2.5, operand=Udh)) <= REL
    F = np.zeros(n)
    Fd = ctx.to_device(F)
    h.lift(Fd, 1.0, 7.5)
    assert relerr(Fd.download(), o.lift(F, 1.0, 7.5)) <= REL


@pytest.mark.parametrize("nsd,nel,hi", [(3, [7, 6, 5], [1, 2, 3]), (2, [9, 7], [1, 2])])
def test_affine_path_matches_quadrature_path(rsd, ctx, monkeypatch, nsd, nel, hi):
    # the same problem on an undistorted mesh: matrix by row gather and vectors one thread per element
    # (default), both by the affine group kernels, and everything by quadrature
    ne = int(np.prod(nel))
    def run():
        h = make_heat(rsd, ctx, nsd, 1, 2, nel, [0] * nsd, hi, k_elem=np.linspace(1, 2, ne), rho=1.5, cp=2.0,
                      dirichlet={0: "0", 3: "1"})
        rng = np.random.default_rng(1)
        U, Ud = ctx.to_device(rng.standard_normal(h.n)), ctx.to_device(rng.standard_normal(h.n))
        h.assemble_matrix(1.0, 4.0)
        out = ctx.array(h.n)
        res = [h.K.values()]
        for which, kw in ((1, dict(U=U)), (2, dict(U=U)), (3, dict(Udot=Ud)), (4, dict(coef=0.5, operand=U))):
            h.assemble_vector(which, out, **kw)
            res.append(out.download())
        F = ctx.to_device(np.zeros(h.n))
        h.lift(F, 1.0, 7.5)
        res.append(F.download())
        return res
    fast = run()
    assert relerr(fast[0], run()[0]) == 0.0   # the matrix gather is deterministic (the vectors use atomics)
    monkeypatch.setenv("RSD_ROW_ASM", "0")
    monkeypatch.setenv("RSD_ELEM_VEC", "0")
    group = run()
    monkeypatch.setenv("RSD_AFFINE", "0")
    quad = run()
    for a, b, c in zip(fast, group, quad):
        assert relerr(a, c) <= 1e-13 and relerr(b, c) <= 1e-13


def test_first_assembly_after_setup(rsd, ctx):
    # the first assembly of a problem builds its lazily made tables (slot map, affine flags and
    # geometry, row adjacency) and must see them complete: a small problem first, then a larger one
    small = make_heat(rsd, ctx, 3, 1, 2, [7, 6, 5], [0, 0, 0], [1, 1, 1], dirichlet={0: "0", 1: "0", 4: "0"})
    small.assemble_matrix(1.0, 50.0)
    bc = {t: "0" for t in range(6)}
    h = make_heat(rsd, ctx, 3, 1, 2, [40, 36, 30], [0, 0, 0], [1, 1, 1], dirichlet=bc)
    h.assemble_matrix(1.0, 50.0)
    o = oracle.Oracle(oracle.BlockMesh(3, [40, 36, 30], [0, 0, 0], [1, 1, 1], 1), 2, bc=bc)
    assert relerr(h.K.values(), o.assemble_matrix(1.0, 50.0)) <= REL


def test_fp32_copy_written_by_row_assembly(rsd, ctx):
    # once a matrix has an FP32 copy, the row-gather assembly writes it alongside the FP64 values;
    # it must equal the copy that converting the FP64 values afresh gives, bit for bit
    bc = {0: "0", 1: "0"}
    h = make_heat(rsd, ctx, 3, 1, 2, [9, 8, 7], [0, 0, 0], [1, 1, 1], dirichlet=bc)
    h.assemble_matrix(1.0, 2.0)
    h.K.sync_f32()
    h.assemble_matrix(1.0, 50.0)
    n = h.n
    x = np.random.default_rng(6).standard_normal(n)
    x32, y32 = ctx.to_device(x.astype(np.float32)), ctx.array(n, np.float32)
    h.K.spmv_f32(x32, y32)
    fused = y32.download()
    v = h.K.values()
    h.K.set_values(v)                  # the same values through CSR: the copy is converted again
    h.K.spmv_f32(x32, y32)
    assert np.array_equal(fused, y32.download())
    rp, col = h.K.pattern()
    o = oracle.Oracle(oracle.BlockMesh(3, [9, 8, 7], [0, 0, 0], [1, 1, 1], 1), 2, bc=bc)
    assert relerr(fused, oracle.spmv(rp, col, o.assemble_matrix(1.0, 50.0), x)) <= 1e-5


def test_steady_cg_and_gmres_match_reference(rsd, ctx):
    h = make_heat(rsd, ctx, 2, 1, 2, [16, 16], [0, 0], [1, 1], dirichlet={t: "(1-x)*(1-y)" for t in range(4)})
    g = golden("steady_q1_quad_16.npz")
    U = ctx.array(h.n).zero()
    rep = h.steady(U, type=rsd.CG, precond=rsd.JACOBI, tol=1e-10, max_iters=1000)
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert relerr(U.download(), g["U"]) <= REL
    g = golden("steady_gmres7_q1_quad_16.npz")
    U.zero()
    rep = h.steady(U, type=rsd.GMRES, precond=rsd.JACOBI, tol=1e-10, max_iters=1000, krylov_dim=7)
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert relerr(U.download(), g["U"]) <= REL


def test_backward_euler_matches_reference(rsd, ctx):
    g = golden("be_q1_hex_6x5x4.npz")
    h = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], rho=1.0, cp=1.0, dirichlet={t: "0" for t in range(6)})
    U, Up = ctx.to_device(g["U0"]), ctx.to_device(g["U0"])
    res = []
    for _ in range(5):
        rep = h.be_step(1e-2, U, Up, type=rsd.CG, precond=rsd.JACOBI, tol=1e-8, max_iters=1000)
        assert rep["converged"]
        res.append(rep["residualNorm"])
    assert relerr(U.download(), g["U"]) <= REL
    assert relerr(res, g["residual"]) <= 1e-9   # norms of residuals ~1e-8 of their parts: cancellation


def test_be_step_with_host_state_matches_device_steps(rsd, ctx):
    # the host-buffer step runs the same kernels on device copies of the state (the right-hand side
    # and residual passes add with atomics, so the last bits may differ between two problems)
    g = golden("be_q1_hex_6x5x4.npz")
    kw = dict(type=rsd.CG, precond=rsd.JACOBI, tol=1e-8, max_iters=1000)
    h1 = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], dirichlet={t: "0" for t in range(6)})
    U, Up = ctx.to_device(g["U0"]), ctx.to_device(g["U0"])
    dev = [h1.be_step(1e-2, U, Up, **kw) for _ in range(5)]
    h2 = make_heat(rsd, ctx, 3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], dirichlet={t: "0" for t in range(6)})
    Uh = np.array(g["U0"], dtype=np.float64)
    host = [h2.be_step_host(1e-2, Uh, **kw) for _ in range(5)]
    assert relerr(Uh, U.download()) <= REL
    assert relerr([r["residualNorm"] for r in host], [r["residualNorm"] for r in dev]) <= 1e-9
    assert all(abs(a["iterations"] - b["iterations"]) <= 1 for a, b in zip(host, dev))
    assert relerr(Uh, g["U"]) <= REL
    with pytest.raises(ValueError):
        h2.be_step_host(1e-2, np.zeros(h2.n, np.float32), **kw)


def test_newton_gmres_matches_reference(rsd, ctx):
    g = golden("newton_q2_hex_3.npz")
    h = make_heat(rsd, ctx, 3, 2, 3, [3, 3, 3], [0, 0, 0], [1, 1, 1], src_expr="10", k_expr="1 + 0.5*T", dk_expr="0.5",
                  dirichlet={0: "0", 1: "1"})
    U = ctx.array(h.n).zero()
    cfg = rsd.SolverConfig.make(type=rsd.GMRES, precond=rsd.JACOBI, tol=1e-12, max_iters=1000, krylov_dim=30)
    rep = h.newton(U, 1e-10, 1e-10, 50, cfg=cfg)
    assert rep["converged"] and rep["iterations"] == g["iterations"]
    assert relerr(U.download(), g["U"]) <= 1e-11


def test_mixed_gmres_and_newton(rsd, ctx):
    # FP32 Arnoldi with FP64 restart residuals: converges on the FP64 residual, and a Newton solve
    # with mixed inner GMRES reaches the FP64 Newton solution
    h = make_heat(rsd, ctx, 3, 2, 3, [6, 5, 4], [0, 0, 0], [1, 1, 1], src_expr="10", k_expr="1 + 0.5*T", dk_expr="0.5",
                  dirichlet={0: "0", 1: "1"})
    U64, Umx = ctx.array(h.n).zero(), ctx.array(h.n).zero()
    r64 = h.newton(U64, 1e-10, 1e-10, 50, cfg=rsd.SolverConfig.make(type=rsd.GMRES, tol=1e-12, max_iters=5000, krylov_dim=30))
    rmx = h.newton(Umx, 1e-10, 1e-10, 50, cfg=rsd.SolverConfig.make(type=rsd.GMRES, precision=rsd.MIXED, tol=1e-12,
                                                                    max_iters=5000, krylov_dim=30))
    assert r64["converged"] and rmx["converged"]
    assert relerr(Umx.download(), U64.download()) <= 1e-9
    # one linear solve with the Jacobian: the reported residual is the FP64 one
    h.assemble_matrix(1.0, 0.0, 1.0, 0.0, U=U64)
    F = ctx.to_device(np.random.default_rng(2).standard_normal(h.n))
    x = ctx.array(h.n).zero()
    rep = rsd.solve(ctx, h.K, F, x, type=rsd.GMRES, precision=rsd.MIXED, tol=1e-10, max_iters=5000, krylov_dim=20)
    rp, col = h.K.pattern()
    r = F.download() - oracle.spmv(rp, col, h.K.values(), x.download())
    assert rep["converged"] and np.linalg.norm(r) / np.linalg.norm(F.download()) < 1e-10
    assert rep["refinements"] >= 1


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_gmres_long_cycles(rsd, ctx, prec):
    # Krylov dimensions past the fused orthogonalization (per-vector CGS passes and a Givens launch of
    # its own beyond 32) and past the shared-memory back substitution (beyond 64 columns): the same
    # solution as GMRES(30), to the FP64-checked tolerance
    h = make_heat(rsd, ctx, 3, 2, 3, [6, 5, 4], [0, 0, 0], [1, 1, 1], src_expr="10", k_expr="1 + 0.5*T", dk_expr="0.5",
                  dirichlet={0: "0", 1: "1"})
    U = ctx.array(h.n)
    U.upload(np.linspace(0.0, 1.0, h.n))
    h.assemble_matrix(1.0, 0.0, 1.0, 0.0, U=U)   # the nonsymmetric Jacobian
    F = ctx.to_device(np.random.default_rng(5).standard_normal(h.n))
    rp, col = h.K.pattern()
    vals = h.K.values()
    precision = rsd.MIXED if prec == "mixed" else rsd.FP64
    sols = {}
    for m in (30, 40, 100):
        x = ctx.array(h.n).zero()
        rep = rsd.solve(ctx, h.K, F, x, type=rsd.GMRES, precision=precision, tol=1e-11, max_iters=5000, krylov_dim=m)
        r = F.download() - oracle.spmv(rp, col, vals, x.download())
        assert rep["converged"] and np.linalg.norm(r) / np.linalg.norm(F.download()) < 1e-11, (m, rep)
        sols[m] = x.download()
    assert relerr(sols[40], sols[30]) < 1e-8 and relerr(sols[100], sols[30]) < 1e-8


def random_csr(n, per_row, seed):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        c = np.unique(np.concatenate([[i], rng.integers(0, n, per_row)]))
        rows.append(c)
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int64)
    val = rng.standard_normal(len(col))
    return rp, col, val


@pytest.mark.parametrize("n,per_row", [(1, 1), (7, 3), (1000, 9), (20000, 27), (5000, 120), (100000, 5)])
def test_spmv_matches_reference(rsd, ctx, n, per_row):
    rp, col, val = random_csr(n, per_row, n)
    A = rsd.CSR.from_host(ctx, rp, col, val)
    x = np.random.default_rng(1).standard_normal(n)
    y_ref = oracle.spmv(rp, col, val, x)
    xd, yd = ctx.to_device(x), ctx.array(n)
    for lanes in (0, 2, 4, 8, 16, 32):
        A.set_launch(lanes, 0)
        A.spmv(xd, yd)
        assert relerr(yd.download(), y_ref) <= 1e-13
    # FP32 values and vector: error bounded by the row's absolute sum times a few FP32 ulps
    bound = 4 * np.finfo(np.float32).eps * oracle.spmv(rp, col, np.abs(val), np.abs(x)) * (rp[1:] - rp[:-1]).max()
    x32, y32 = ctx.to_device(x.astype(np.float32)), ctx.array(n, np.float32)
    for lanes in (0, 4):
        A.set_launch(lanes, 0)
        A.sync_f32()
        A.spmv_f32(x32, y32)
        assert (np.abs(y32.download() - y_ref) <= bound + 1e-30).all()


def test_layouts_stay_in_step(rsd, ctx):
    # Values live in CSR (API order) and SELL-32 (execution order); every write through one layout
    # must be seen through the other, in FP64 and in the FP32 copy.
    h = make_heat(rsd, ctx, 3, 1, 2, [9, 7, 5], [0, 0, 0], [1, 1, 1], dirichlet={0: "0", 1: "0"})
    m = oracle.BlockMesh(3, [9, 7, 5], [0, 0, 0], [1, 1, 1], 1)
    o = oracle.Oracle(m, 2, bc={0: "0", 1: "0"})
    rp, col = h.K.pattern()
    n = h.n
    h.assemble_matrix(1.0, 3.0)                      # scatter lands in SELL
    v = o.assemble_matrix(1.0, 3.0)
    x = np.random.default_rng(4).standard_normal(n)
    xd, yd = ctx.to_device(x), ctx.array(n)
    for lanes in (0, 4):
        h.K.set_launch(lanes, 0)
        h.K.spmv(xd, yd)
        assert relerr(yd.download(), oracle.spmv(rp, col, v, x)) <= REL
    assert relerr(h.K.values(), v) <= REL          # SELL -> CSR
    h.K.set_values(2.0 * v)                          # CSR -> SELL
    d = ctx.array(n)
    for lanes in (0, 8):
        h.K.set_launch(lanes, 0)
        h.K.spmv(xd, yd)
        assert relerr(yd.download(), oracle.spmv(rp, col, 2.0 * v, x)) <= REL
        h.K.diagonal(d)
        dia = np.array([v[rp[i]:rp[i + 1]][col[rp[i]:rp[i + 1]] == i][0] for i in range(n)])
        assert relerr(d.download(), 2.0 * dia) == 0.0
        h.K.lump(d)
        assert relerr(d.download(), 2.0 * np.add.reduceat(v, rp[:-1])) <= REL
        # the FP32 copy follows the FP64 values and the layout
        h.K.sync_f32()
        x32, y32 = ctx.to_device(x.astype(np.float32)), ctx.array(n, np.float32)
        h.K.spmv_f32(x32, y32)
        assert relerr(y32.download(), oracle.spmv(rp, col, 2.0 * v, x)) <= 1e-5
    h.K.set_launch(0, 0)
    lanes, block, us = h.K.autotune()
    assert lanes in (0, 2, 4, 8, 16, 32) and block in (128, 256, 512) and us > 0
    h.K.spmv(xd, yd)
    assert relerr(yd.download(), oracle.spmv(rp, col, 2.0 * v, x)) <= REL


def test_blas1_matches_numpy(rsd, ctx):
    rng = np.random.default_rng(3)
    n = 100003
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    xd, yd = ctx.to_device(x), ctx.to_device(y)
    import ctypes as C
    out = C.c_double()
    rsd.check(rsd.lib().rsd_dot(ctx.h, n, xd.ptr, yd.ptr, C.byref(out)))
    assert abs(out.value - x @ y) <= 1e-12 * np.abs(x * y).sum()
    rsd.check(rsd.lib().rsd_axpby(ctx.h, n, 2.0, -0.5, xd.ptr, yd.ptr))
    assert relerr(yd.download(), -0.5 * y + 2.0 * x) <= 1e-15
    rsd.check(rsd.lib().rsd_mul(ctx.h, n, xd.ptr, xd.ptr, yd.ptr))
    assert relerr(yd.download(), x * x) == 0.0
    rsd.check(rsd.lib().rsd_nrm2(ctx.h, n, xd.ptr, C.byref(out)))
    assert abs(out.value - np.linalg.norm(x)) <= 1e-12 * np.linalg.norm(x)
    rsd.check(rsd.lib().rsd_dot(ctx.h, 0, xd.ptr, yd.ptr, C.byref(out)))
    assert out.value == 0.0


def test_krylov_known_answers(rsd, ctx):
    # cg/Solver.cpp:12-68 and gmres/Solver.cpp:12-172 of the reference's unit tests
    A = rsd.CSR.from_host(ctx, [0, 2, 4], [0, 1, 0, 1], [4.0, 1.0, 1.0, 3.0])
    b, x = ctx.to_device(np.array([1.0, 2.0])), ctx.array(2).zero()
    rep = rsd.solve(ctx, A, b, x, type=rsd.CG, tol=1e-12)
    assert rep["converged"] and np.allclose(x.download(), [1 / 11, 7 / 11], atol=1e-10)
    B = rsd.CSR.from_host(ctx, [0, 2, 4], [0, 1, 0, 1], [2.0, 1.0, 3.0, 4.0])
    b2, x2 = ctx.to_device(np.array([1.0, 3.0])), ctx.array(2).zero()
    rep = rsd.solve(ctx, B, b2, x2, type=rsd.GMRES, krylov_dim=1, tol=1e-10, max_iters=200)
    assert rep["converged"] and np.allclose(x2.download(), [0.2, 0.6], atol=1e-8)


def test_mixed_precision_reaches_fp64_checked_tolerance(rsd, ctx):
    h = make_heat(rsd, ctx, 3, 1, 2, [24, 24, 24], [0, 0, 0], [1, 1, 1], src_expr="1", dirichlet={t: "0" for t in range(6)})
    n = h.n
    h.assemble_matrix(1.0, 1000.0)
    F = ctx.array(n)
    h.assemble_vector(0, F)
    x64, xmx = ctx.array(n).zero(), ctx.array(n).zero()
    r64 = rsd.solve(ctx, h.K, F, x64, type=rsd.CG, tol=1e-8)
    rmx = rsd.solve(ctx, h.K, F, xmx, type=rsd.CG, precision=rsd.MIXED, tol=1e-8)
    assert r64["converged"] and rmx["converged"] and rmx["refinements"] >= 1
    assert rmx["trueResidualRel"] < 1e-8          # checked in FP64 with the FP64 matrix
    assert r64["trueResidualRel"] < 1.01e-8
    # stated error against the FP64 solve: both within tol * cond of the exact solution
    assert relerr(xmx.download(), x64.download()) < 1e-6


def test_graph_solve_matches_plain_launches(rsd, ctx, monkeypatch):
    # The CG solve runs as one CUDA graph (device-side WHILE loop, IF node for the FP64 residual
    # replacement); the plain launch sequence runs the same kernels, so both give the same iterates.
    h = make_heat(rsd, ctx, 3, 1, 2, [30, 26, 22], [0, 0, 0], [1, 1, 1], src_expr="1 + x", dirichlet={0: "0", 2: "y"})
    n = h.n
    h.assemble_matrix(1.0, 200.0)
    F = ctx.array(n)
    h.assemble_vector(0, F)
    for prec in (rsd.FP64, rsd.MIXED):
        outs = []
        for mode in ("1", "0", "1"):            # graph, plain, graph again (cached graph reused)
            monkeypatch.setenv("RSD_CG_GRAPH", mode)
            x = ctx.array(n).zero()
            rep = rsd.solve(ctx, h.K, F, x, type=rsd.CG, precision=prec, tol=1e-9, max_iters=5000)
            assert rep["converged"]
            outs.append((rep["iterations"], rep["trueResidualRel"], x.download()))
        for it, tr, xv in outs[1:]:
            assert it == outs[0][0] and tr == outs[0][1] and np.array_equal(xv, outs[0][2])
        # a different right-hand side buffer rebuilds the graph; the answer follows the new b
        G = ctx.to_device(2.0 * F.download())
        x2 = ctx.array(n).zero()
        monkeypatch.setenv("RSD_CG_GRAPH", "1")
        rep = rsd.solve(ctx, h.K, G, x2, type=rsd.CG, precision=prec, tol=1e-9, max_iters=5000)
        assert rep["converged"] and relerr(x2.download(), 2.0 * outs[0][2]) < 1e-6
    # max_iters reached inside the graph: not converged, iteration count as the plain path reports
    for mode in ("1", "0"):
        monkeypatch.setenv("RSD_CG_GRAPH", mode)
        x = ctx.array(n).zero()
        rep = rsd.solve(ctx, h.K, F, x, type=rsd.CG, tol=1e-14, max_iters=7)
        assert not rep["converged"] and rep["iterations"] == 7


def test_edge_cases(rsd, ctx):
    # empty matrix
    E = rsd.CSR.from_host(ctx, [0], [], [])
    assert E.n == 0
    rep = rsd.solve(ctx, E, None, None, type=rsd.CG)
    assert rep["converged"]
    # maxIters = 1: no iteration runs (cg/Solver.tpp:66), not converged
    A = rsd.CSR.from_host(ctx, [0, 2, 4], [0, 1, 0, 1], [4.0, 1.0, 1.0, 3.0])
    b, x = ctx.to_device(np.array([1.0, 2.0])), ctx.array(2).zero()
    rep = rsd.solve(ctx, A, b, x, type=rsd.CG, tol=1e-12, max_iters=1)
    assert not rep["converged"] and rep["iterations"] == 1
    # Jacobi with a (near) zero diagonal uses 1 (Jacobi.hpp:33)
    Z = rsd.CSR.from_host(ctx, [0, 1, 2], [0, 1], [1e-320, 2.0])
    d = ctx.array(2)
    Z.jacobi(d)
    assert (d.download() == [1.0, 0.5]).all()
    # NaN in the right-hand side comes back as a status, not a hang
    bn, xn = ctx.to_device(np.array([np.nan, 1.0])), ctx.array(2).zero()
    rep = rsd.solve(ctx, A, bn, xn, type=rsd.CG, tol=1e-12, max_iters=50)
    assert not rep["converged"] and rep["status"] in (-5, -6)
    # invalid arguments are errors
    with pytest.raises(rsd.RsdError):
        rsd.CSR.from_host(ctx, [0, 2], [0, 5], [1.0, 1.0])
    xyz, ien, rng = bm().block_mesh(2, [2, 2], [0, 0], [1, 1], 1)
    mesh = rsd.Mesh(ctx, 2, 1, xyz, ien, rng)
    with pytest.raises(rsd.RsdError) as e:
        rsd.Heat(ctx, mesh, 2, src_expr="not an expression (")
    assert e.value.code == -7
    with pytest.raises(rsd.RsdError):
        rsd.Heat(ctx, mesh, 7)
    with pytest.raises(rsd.RsdError):
        xyz3, ien3, rng3 = bm().block_mesh(3, [1, 1, 1], [0, 0, 0], [1, 1, 1], 3)
        rsd.Mesh(ctx, 3, 3, xyz3, ien3, rng3)       # Q3 hex: 64 nodes per element, unsupported


def test_larger_case_against_restatement(rsd, ctx):
    # 20^3 Q1 hex: pattern bit-exact and values within 1e-12 of the restatement
    m = oracle.BlockMesh(3, [20, 20, 20], [0, 0, 0], [1, 1, 1], 1)
    o = oracle.Oracle(m, 2, src_expr="1", bc={t: "0" for t in range(6)})
    h = make_heat(rsd, ctx, 3, 1, 2, [20, 20, 20], [0, 0, 0], [1, 1, 1], src_expr="1", dirichlet={t: "0" for t in range(6)})
    rp, col = h.K.pattern()
    orp, ocol = o.pattern()
    assert (rp == orp).all() and (col == ocol).all()
    h.assemble_matrix(1.0, 1000.0)
    v = o.assemble_matrix(1.0, 1000.0)
    assert relerr(h.K.values(), v) <= REL
    F = ctx.array(h.n)
    h.assemble_vector(0, F)
    assert relerr(F.download(), o.assemble_vector(0)) <= REL
    # grid lines of 19 rows: most slices hold a line end, whose rows miss neighbours of the slice's
    # stencil pattern (zeros in the execution layout); products, diagonal and FP32 copy see none of it
    x = np.random.default_rng(8).standard_normal(h.n)
    xd, yd, d = ctx.to_device(x), ctx.array(h.n), ctx.array(h.n)
    h.K.spmv(xd, yd)
    assert relerr(yd.download(), oracle.spmv(rp, col, v, x)) <= REL
    h.K.diagonal(d)
    vd = h.K.values()
    assert relerr(d.download(), np.array([vd[rp[i]:rp[i + 1]][col[rp[i]:rp[i + 1]] == i][0] for i in range(h.n)])) == 0.0
    h.K.sync_f32()
    x32, y32 = ctx.to_device(x.astype(np.float32)), ctx.array(h.n, np.float32)
    h.K.spmv_f32(x32, y32)
    assert relerr(y32.download(), oracle.spmv(rp, col, v, x)) <= 1e-5


@pytest.mark.parametrize("nx,ny", [(50, 37), (32, 8), (7, 40)])
def test_spmv_grid_with_line_ends(rsd, ctx, nx, ny):
    # 9-point stencil on an nx x ny grid with no boundary rows removed: rows at line ends and on the
    # first and last lines miss neighbours, and rows near both ends of the matrix have offsets that
    # would leave [0, n) -- the layout must keep those slices apart
    n = nx * ny
    rows = []
    for j in range(ny):
        for i in range(nx):
            rows.append(sorted((j + b) * nx + (i + a) for b in (-1, 0, 1) for a in (-1, 0, 1)
                               if 0 <= i + a < nx and 0 <= j + b < ny))
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int64)
    val = np.random.default_rng(nx).standard_normal(len(col))
    A = rsd.CSR.from_host(ctx, rp, col, val)
    x = np.random.default_rng(ny).standard_normal(n)
    xd, yd = ctx.to_device(x), ctx.array(n)
    A.spmv(xd, yd)
    assert relerr(yd.download(), oracle.spmv(rp, col, val, x)) <= 1e-13
    assert relerr(A.values(), val) == 0.0
    A.set_values(2.0 * val)
    A.spmv(xd, yd)
    assert relerr(yd.download(), oracle.spmv(rp, col, 2.0 * val, x)) <= 1e-13


def test_size_independent_properties_at_scale(rsd, ctx):
    # 96^3 Q1 hex (857k rows): K + M/dt is symmetric with positive diagonal, SpMV is linear,
    # K.1 vanishes on rows away from the Dirichlet boundary
    h = make_heat(rsd, ctx, 3, 1, 2, [96, 96, 96], [0, 0, 0], [1, 1, 1], dirichlet={t: "0" for t in range(6)})
    n = h.n
    h.assemble_matrix(1.0, 0.0)
    rng = np.random.default_rng(5)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    xd, yd, zd = ctx.to_device(x), ctx.to_device(y), ctx.to_device(x + 2 * y)
    ax, ay, az = ctx.array(n), ctx.array(n), ctx.array(n)
    h.K.spmv(xd, ax); h.K.spmv(yd, ay); h.K.spmv(zd, az)
    assert relerr(az.download(), ax.download() + 2 * ay.download()) < 1e-12
    ones, k1 = ctx.to_device(np.ones(n)), ctx.array(n)
    h.K.spmv(ones, k1)
    t2a, a2t = h.dofmap()
    ijk = np.stack(np.unravel_index(a2t, (97, 97, 97)), 1)
    interior = ((ijk >= 2) & (ijk <= 94)).all(1)
    assert np.abs(k1.download()[interior]).max() < 1e-12
    # symmetry via x.Ay == y.Ax
    assert abs(x @ ay.download() - y @ ax.download()) < 1e-10 * abs(x @ ax.download())


def test_time_dependent_dirichlet_values(rsd, ctx):
    # Dirichlet expressions of t and x evaluated on the device at each step's time (and at t - dt for
    # the mass right-hand side) against the restatement's host evaluation
    bc = {0: "sin(3*t + x) + y", 1: "t*y", 3: "0.25"}
    m = oracle.BlockMesh(2, [9, 7], [0, 0], [1, 1], 2)
    o = oracle.Oracle(m, 3, bc=bc, src_expr="1 + t")
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 2, 2, m.xyz, m.ien, m.rng), 3, src_expr="1 + t", dirichlet=bc)
    U0 = np.sin(np.arange(o.n) * 0.11)
    Uo, reso, _, _ = o.backward_euler(0.04, 5, U0, tol=1e-11)
    U, Up = ctx.to_device(U0), ctx.to_device(U0)
    res = [h.be_step(0.04, U, Up, type=rsd.CG, precond=rsd.JACOBI, tol=1e-11)["residualNorm"] for _ in range(5)]
    assert relerr(U.download(), Uo) <= REL
    assert relerr(res, reso) <= 1e-9


def test_sorted_slice_layout_matches_natural_layout(rsd, ctx, monkeypatch):
    """RSD_SELL_SORT=1 lays a Q2 matrix's slices out by row kind (SELL-C-sigma): fewer padded slots,
    the same assembled values, bit-identical SpMV rows, and CG (FP64 and the persistent mixed kernel)
    and GMRES solutions equal to the natural layout's to rounding."""
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("RSD_SELL_SORT", mode)
        h = make_heat(rsd, ctx, 3, 2, 3, [8, 7, 6], [0, 0, 0], [1, 1, 1], src_expr="10", dirichlet={0: "0", 1: "1"})
        h.assemble_matrix(1.0, 5.0)
        n = h.n
        x = ctx.to_device(np.cos(np.arange(n) * 0.7))
        y = ctx.array(n)
        h.K.spmv(x, y)
        F = ctx.array(n)
        h.assemble_vector(0, F)
        sols = {}
        for key, kw in (("cg64", dict(type=rsd.CG)), ("cgmx", dict(type=rsd.CG, precision=rsd.MIXED)),
                        ("gmres", dict(type=rsd.GMRES, krylov_dim=30))):
            u = ctx.array(n).zero()
            rep = rsd.solve(ctx, h.K, F, u, tol=1e-11, max_iters=5000, **kw)
            assert rep["converged"], (mode, key)
            sols[key] = (rep["iterations"], u.download())
        out[mode] = (h.K.layout(), h.K.values(), y.download(), sols)
    (lay0, v0, y0, s0), (lay1, v1, y1, s1) = out["0"], out["1"]
    assert lay1["sell_slots"] < 0.8 * lay0["sell_slots"]
    assert relerr(v1, v0) <= 1e-13
    assert np.array_equal(y1, y0) or relerr(y1, y0) <= 1e-15
    for key in s0:
        assert abs(s1[key][0] - s0[key][0]) <= 2, key
        assert relerr(s1[key][1], s0[key][1]) <= 1e-9, key


def test_mirrored_slices_give_the_same_mixed_solve(rsd, ctx, monkeypatch):
    """The row-gather assembly of 8-node elements writes K + M/dt symmetric to the last bit; the mixed
    CG's FP32 SpMV then reads the negative-offset entries of mirrored stencil slices from the mirror
    rows.  Same row sums in the same order: the solve equals the whole-row one bit for bit.  A write
    that is not known symmetric turns the mirrored reads off."""
    h = make_heat(rsd, ctx, 3, 1, 2, [20, 18, 16], [0, 0, 0], [1, 1, 1], src_expr="1 + x*y",
                  k_elem=np.exp(np.sin(np.arange(20 * 18 * 16))), dirichlet={t: "0" for t in range(6)})
    h.assemble_matrix(1.0, 1.0 / 1e-3)
    lay = h.K.layout()
    assert lay["mirrored_slices"] > 0.5 * lay["slices"] and lay["mirrored_active"]
    F = ctx.array(h.n)
    h.assemble_vector(0, F)
    outs = []
    for sym in ("1", "0"):
        monkeypatch.setenv("RSD_SYM_SPMV", sym)
        for persist in ("1", "0"):
            monkeypatch.setenv("RSD_CG_PERSIST", persist)
            x = ctx.array(h.n).zero()
            rep = rsd.solve(ctx, h.K, F, x, type=rsd.CG, precision=rsd.MIXED, tol=1e-10, max_iters=5000)
            assert rep["converged"]
            outs.append((rep["iterations"], x.download()))
    for it, xv in outs[1:]:
        assert it == outs[0][0] and np.array_equal(xv, outs[0][1])
    # values written through the CSR view are not known symmetric: the whole rows are read again
    h.K.set_values(h.K.values())
    assert not h.K.layout()["mirrored_active"]
    monkeypatch.setenv("RSD_SYM_SPMV", "1")
    x = ctx.array(h.n).zero()
    rep = rsd.solve(ctx, h.K, F, x, type=rsd.CG, precision=rsd.MIXED, tol=1e-10, max_iters=5000)
    assert rep["converged"] and rep["iterations"] == outs[0][0] and np.array_equal(x.download(), outs[0][1])
