"""GPU checks of the adjoint pair (rsd_heat_forward / rsd_heat_backward).

The gradient of J = 0.5 ||T(theta) - T_obs||^2 with k_e = exp(theta_e) is compared with
  * the golden fixture made by the reference's own templates (oracle/_ref: forward and adjoint
    solves by the reference CG, element gradient by the reference DiffusionForm), <= 1e-9 relative;
  * central finite differences of J through the device forward solve (h = 1e-6), <= 1e-6 relative;
  * the FP64 CPU adjoint of the C restatement, <= 1e-9 relative.
"""
from importlib import import_module

import numpy as np
import pytest

import oracle
from conftest import golden

pytestmark = pytest.mark.gpu
TIGHT = dict(tol=1e-14, max_iters=100000)


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make_heat(rsd, ctx, nel, dirichlet, src="1"):
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rng = bm.block_mesh(3, nel, [0, 0, 0], [1, 1, 1], 1)
    mesh = rsd.Mesh(ctx, 3, 1, xyz, ien, rng)
    return rsd.Heat(ctx, mesh, 2, src_expr=src, dirichlet=dirichlet), xyz, ien


def test_adjoint_matches_reference_fixture(rsd, ctx):
    g = golden("adjoint_q1_hex_6x5x4.npz")
    bc = {t: "0" for t in range(6)}
    bc[1] = "0.5"
    h, _, _ = make_heat(rsd, ctx, [6, 5, 4], bc)
    theta = ctx.to_device(g["theta"])
    T = ctx.array(h.n).zero()
    rep = h.forward(theta, T, **TIGHT)
    assert rep["converged"]
    assert relerr(T.download(), g["T"]) <= 1e-11
    dJdT = ctx.to_device(T.download() - g["Tobs"])
    grad = ctx.array(g["theta"].size)
    rep = h.backward(theta, T, dJdT, grad, **TIGHT)
    assert rep["converged"]
    assert relerr(grad.download(), g["grad"]) <= 1e-9
    assert abs(grad.download() @ g["fd_dir"] - g["fd"]) <= 1e-6 * abs(g["fd"])


def fourier_theta(xyz, ien, modes=8, seed=5):
    rng = np.random.default_rng(seed)
    c = xyz.reshape(-1, 3)[ien.reshape(len(ien) // 8 if ien.ndim == 1 else ien.shape[0], -1)].mean(axis=1)
    th = np.zeros(len(c))
    for _ in range(modes):
        k = rng.integers(1, 5, 3)
        th += 0.5 * np.sin(2 * np.pi * (c @ k) + rng.uniform(0, 2 * np.pi))
    return th / np.sqrt(modes)


def test_adjoint_matches_finite_differences_and_cpu_adjoint(rsd, ctx):
    nel = [14, 12, 10]
    h, xyz, ien = make_heat(rsd, ctx, nel, {t: "0" for t in range(6)})
    theta_h = fourier_theta(xyz, ien)
    obs_h = fourier_theta(xyz, ien, seed=55)
    ne, n = theta_h.size, h.n
    theta = ctx.to_device(theta_h)
    # observations: the forward solution of a second theta
    Tobs = ctx.array(n).zero()
    h.forward(ctx.to_device(obs_h), Tobs, **TIGHT)
    Tobs_h = Tobs.download()
    T = ctx.array(n).zero()
    h.forward(theta, T, **TIGHT)
    T_h = T.download()
    grad = ctx.array(ne)
    h.backward(theta, T, ctx.to_device(T_h - Tobs_h), grad, **TIGHT)
    grad_h = grad.download()

    def J(th):
        Tt = ctx.array(n).zero()
        h.forward(ctx.to_device(th), Tt, **TIGHT)
        return 0.5 * np.sum((Tt.download() - Tobs_h) ** 2)

    rng = np.random.default_rng(555)
    for _ in range(4):
        d = rng.standard_normal(ne)
        d /= np.linalg.norm(d)
        fd = (J(theta_h + 1e-6 * d) - J(theta_h - 1e-6 * d)) / 2e-6
        assert abs(fd - grad_h @ d) <= 1e-6 * abs(fd)
    # FP64 CPU adjoint of the restatement on the same theta and observations
    m = oracle.BlockMesh(3, nel, [0, 0, 0], [1, 1, 1], 1)
    o = oracle.Oracle(m, 2, k_elem=np.exp(theta_h), src_expr="1", bc={t: "0" for t in range(6)})
    To, _ = o.steady(0, 1, 1e-14, 100000)
    assert relerr(To, T_h) <= 1e-10
    rp, col = o.pattern()
    lam, _ = oracle.csr_solve(rp, col, o.assemble_matrix(1.0), To - Tobs_h, tol=1e-14, maxit=100000)
    g_cpu = -np.exp(theta_h) * o.adjoint_gradient(To, lam)
    assert relerr(grad_h, g_cpu) <= 1e-9


def test_autograd_function(rsd, ctx):
    torch = pytest.importorskip("torch")
    HeatSolve = import_module("residuum_solver_b200.autograd").HeatSolve
    h, xyz, ien = make_heat(rsd, ctx, [8, 7, 6], {t: "0" for t in range(6)})
    theta = torch.tensor(fourier_theta(xyz, ien), dtype=torch.float64, device="cuda", requires_grad=True)
    Tobs = torch.linspace(0, 0.01, h.n, dtype=torch.float64, device="cuda")
    cfg = rsd.SolverConfig.make(**TIGHT)
    T = HeatSolve.apply(theta, h, cfg)
    J = 0.5 * ((T - Tobs) ** 2).sum()
    J.backward()
    grad = ctx.array(theta.numel())
    h.backward(theta.detach(), T.detach(), (T - Tobs).detach(), grad, cfg)
    assert relerr(theta.grad.cpu().numpy(), grad.download()) <= 1e-12
