"""rsd_cg_solve_static: FP64 CG over a file-scope device scratch, allocating nothing.

Compared with rsd_solve's FP64 CG (same kernels, grids and reductions, so the same iterates bit for
bit) on two calls in a row, which also checks that each call clears the scratch state the previous
one left (reduction tickets, done/converged flags).  Collected last so that it runs both alone and
after every other GPU test in one process.
"""
from importlib import import_module

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 18


def _heat(rsd, ctx, nel):
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rng = bm.block_mesh(3, nel, [0, 0, 0], [1, 1, 1], 1)
    mesh = rsd.Mesh(ctx, 3, 1, xyz, ien, rng)
    return rsd.Heat(ctx, mesh, 2, src_expr="1 + x*y", dirichlet={0: "0", 1: "x", 4: "0"})


def test_static_cg_matches_solve_on_two_calls(rsd, ctx):
    h = _heat(rsd, ctx, [40, 36, 30])            # 41*37*31 nodes, 45,880 free rows
    n = h.n
    assert n <= MAX_ROWS
    h.assemble_matrix(1.0, 50.0)
    F = ctx.array(n)
    h.assemble_vector(0, F)
    rhs = [F.download(), np.random.default_rng(11).standard_normal(n)]
    for precond in (rsd.JACOBI, rsd.IDENTITY):
        for b_host in rhs:                       # two calls in a row on the same scratch
            b = ctx.to_device(b_host)
            x_ref, x_st = ctx.array(n).zero(), ctx.array(n).zero()
            r_ref = rsd.solve(ctx, h.K, b, x_ref, type=rsd.CG, precond=precond, tol=1e-10, max_iters=2000)
            r_st = rsd.solve_static(ctx, h.K, b, x_st, type=rsd.CG, precond=precond, tol=1e-10, max_iters=2000)
            assert r_ref["converged"] and r_st["converged"]
            assert r_st["iterations"] == r_ref["iterations"]
            assert r_st["finalResidual"] == r_ref["finalResidual"]
            assert r_st["trueResidualRel"] == r_ref["trueResidualRel"]
            assert np.array_equal(x_st.download(), x_ref.download())


def test_static_cg_limits(rsd, ctx):
    # one row more than the scratch holds: rejected with a message, nothing launched
    n = MAX_ROWS + 1
    rp = np.arange(n + 1, dtype=np.int64)
    A = rsd.CSR.from_host(ctx, rp, np.arange(n, dtype=np.int64), np.full(n, 2.0))
    b, x = ctx.array(n).zero(), ctx.array(n).zero()
    with pytest.raises(rsd.RsdError) as e:
        rsd.solve_static(ctx, A, b, x, type=rsd.CG)
    assert e.value.code == -1 and "262144" in str(e.value)
    # exactly at the limit: solved
    n = MAX_ROWS
    A = rsd.CSR.from_host(ctx, np.arange(n + 1, dtype=np.int64), np.arange(n, dtype=np.int64), np.full(n, 2.0))
    b, x = ctx.to_device(np.ones(n)), ctx.array(n).zero()
    rep = rsd.solve_static(ctx, A, b, x, type=rsd.CG, precond=rsd.IDENTITY, tol=1e-12)
    assert rep["converged"] and np.allclose(x.download(), 0.5, rtol=0, atol=1e-14)
    # only FP64 CG
    with pytest.raises(rsd.RsdError):
        rsd.solve_static(ctx, A, b, x, type=rsd.GMRES)
    with pytest.raises(rsd.RsdError):
        rsd.solve_static(ctx, A, b, x, type=rsd.CG, precision=rsd.MIXED)
