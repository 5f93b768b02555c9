"""GPU checks of the batched persistent solver (rsd_batch_*): uneven 2D problems with per-element
log-normal conductivity, solved together in one launch, against single-system solves and the
reference's own CG (oracle/_ref, when built) problem by problem."""
from importlib import import_module

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make_problems(rsd, ctx, count, seed=3, lo=6, hi=48):
    bm = import_module("residuum_solver_b200.blockmesh")
    rng = np.random.default_rng(seed)
    probs = []
    for _ in range(count):
        nx, ny = (int(v) for v in rng.integers(lo, hi + 1, 2))
        xyz, ien, rg = bm.block_mesh(2, [nx, ny], [0, 0], [1, 1], 1)
        ke = np.exp(rng.standard_normal(nx * ny))
        h = rsd.Heat(ctx, rsd.Mesh(ctx, 2, 1, xyz, ien, rg), 2, k_elem=ke, src_expr="1",
                     dirichlet={t: "0" for t in range(4)})
        h.assemble_matrix(1.0)
        F = ctx.array(h.n)
        h.assemble_vector(0, F)
        probs.append((h, F, nx, ny, ke))
    return probs


def true_rel(h, F, x):
    rp, col = h.K.pattern()
    v = h.K.values()
    b = F.download()
    r = b - oracle.spmv(rp, col, v, x)
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_batch_matches_single_solves(rsd, ctx, prec):
    probs = make_problems(rsd, ctx, 24)
    precision = rsd.MIXED if prec == "mixed" else rsd.FP64
    cfg = rsd.SolverConfig.make(precision=precision, tol=1e-8, max_iters=20000)
    B = rsd.Batch(ctx, [h.K for h, *_ in probs])
    xs = [ctx.array(h.n).zero() for h, *_ in probs]
    reps = B.solve([F for _, F, *_ in probs], xs, cfg)
    for (h, F, *_), x, rep in zip(probs, xs, reps):
        assert rep["converged"], rep
        xb = x.download()
        # the FP64-checked relative residual (x0 = 0, so ||r0|| = ||b||)
        assert true_rel(h, F, xb) < (1e-8 if prec == "mixed" else 1.0000001e-8)
        xs1 = ctx.array(h.n).zero()
        r1 = rsd.solve(ctx, h.K, F, xs1, rsd.SolverConfig.make(tol=1e-8, max_iters=20000))
        assert relerr(xb, xs1.download()) < 1e-6
        if prec == "fp64":
            # same algorithm, different reduction order (block sums here, grid sums there), on a right-
            # hand side assembled with atomics: on these ill-conditioned problems rounding can move
            # the iteration where the 1e-8 threshold is crossed by a step or two
            assert abs(rep["iterations"] - r1["iterations"]) <= max(2, 0.02 * r1["iterations"])
    # a second solve on the same batch (the queue and reports reset)
    xs2 = [ctx.array(h.n).zero() for h, *_ in probs]
    reps2 = B.solve([F for _, F, *_ in probs], xs2, cfg)
    for x, x2, r, r2 in zip(xs, xs2, reps, reps2):
        assert r2["iterations"] == r["iterations"] and np.array_equal(x.download(), x2.download())


def test_batch_against_reference_cg(rsd, ctx):
    if not oracle.reference_available():
        pytest.skip("oracle/_ref not built")
    probs = make_problems(rsd, ctx, 6, seed=11, lo=8, hi=30)
    B = rsd.Batch(ctx, [h.K for h, *_ in probs])
    xs = [ctx.array(h.n).zero() for h, *_ in probs]
    reps = B.solve([F for _, F, *_ in probs], xs, rsd.SolverConfig.make(precision=rsd.FP64, tol=1e-10, max_iters=20000))
    for (h, F, *_), x, rep in zip(probs, xs, reps):
        rp, col = h.K.pattern()
        xr, rr = oracle.ref_csr_solve(rp, col, h.K.values(), F.download(), tol=1e-10, maxit=20000)
        assert rr["converged"] and rep["converged"]
        assert abs(rep["iterations"] - rr["iterations"]) <= 1
        assert relerr(x.download(), xr) < 1e-8


def test_batch_edge_cases(rsd, ctx):
    # an empty system and a 1x1 system beside a regular one; max_iters reached is reported
    E = rsd.CSR.from_host(ctx, [0], [], [])
    O = rsd.CSR.from_host(ctx, [0, 1], [0], [4.0])
    probs = make_problems(rsd, ctx, 1, seed=5)
    h, F = probs[0][0], probs[0][1]
    B = rsd.Batch(ctx, [E, O, h.K])
    b1 = ctx.to_device(np.array([2.0]))
    xs = [ctx.array(1).zero(), ctx.array(1).zero(), ctx.array(h.n).zero()]
    reps = B.solve([ctx.array(1).zero(), b1, F], xs, precision=rsd.MIXED, tol=1e-10, max_iters=5000)
    assert reps[0]["converged"] and reps[1]["converged"] and reps[2]["converged"]
    assert abs(xs[1].download()[0] - 0.5) < 1e-12
    reps = B.solve([ctx.array(1).zero(), b1, F], [ctx.array(1).zero(), ctx.array(1).zero(), ctx.array(h.n).zero()],
                   precision=rsd.FP64, tol=1e-14, max_iters=3)
    assert not reps[2]["converged"] and reps[2]["iterations"] == 3
    with pytest.raises(rsd.RsdError):
        B.solve([None, b1, F], xs)


@pytest.mark.parametrize("prec,team", [("mixed", None), ("fp64", None), ("mixed", "2"), ("mixed", "4"), ("fp64", "8")])
def test_team_and_single_cta_paths_agree(rsd, ctx, prec, team, monkeypatch):
    # teams of CTAs per problem (the size chosen for the batch, or forced by RSD_BATCH_TEAM) and one
    # CTA per problem (RSD_BATCH_TEAM=0) run the same PCG with a different reduction order: same
    # convergence, solutions within the tolerance
    probs = make_problems(rsd, ctx, 12, seed=21)
    precision = rsd.MIXED if prec == "mixed" else rsd.FP64
    cfg = rsd.SolverConfig.make(precision=precision, tol=1e-9, max_iters=20000)
    B = rsd.Batch(ctx, [h.K for h, *_ in probs])
    runs = []
    for env in (team, "0"):
        if env is None:
            monkeypatch.delenv("RSD_BATCH_TEAM", raising=False)
        else:
            monkeypatch.setenv("RSD_BATCH_TEAM", env)
        xs = [ctx.array(h.n).zero() for h, *_ in probs]
        reps = B.solve([F for _, F, *_ in probs], xs, cfg)
        runs.append(([x.download() for x in xs], reps))
    for (h, F, *_), xa, xb, ra, rb in zip(probs, runs[0][0], runs[1][0], runs[0][1], runs[1][1]):
        assert ra["converged"] and rb["converged"]
        assert true_rel(h, F, xa) < 1.0000001e-9 and true_rel(h, F, xb) < 1.0000001e-9
        assert abs(ra["iterations"] - rb["iterations"]) <= max(2, 0.02 * rb["iterations"])
        assert relerr(xa, xb) < 1e-6
