"""GPU checks of the transient adjoint pair (rsd_heat_transient_forward / rsd_heat_transient_backward):
7 Backward-Euler steps on a 6x5x4 Q1 mesh with k_e = exp(theta_e), J = 0.5 ||U_7 - U_obs||^2, against
  * the FP64 CPU adjoint on the reference's own templates (fixture), <= 1e-9 relative;
  * central differences of J through the device's forward steps (h = 1e-6, 20 directions), <= 1e-6;
  * the states held: ceil(7 / 3) checkpoints + a segment of 3 + 1 = 7, about 2 sqrt(N), not N;
  * the torch autograd Function over the pair.
"""
import math
from importlib import import_module

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
TIGHT = dict(tol=1e-14, max_iters=100000)


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make(rsd, ctx):
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rng = bm.block_mesh(3, [6, 5, 4], [0, 0, 0], [1, 1, 1], 1)
    bc = {t: "0" for t in range(6)}
    bc[1] = "0.5"
    return rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, xyz, ien, rng), 2, src_expr="1", dirichlet=bc)


def test_transient_adjoint_matches_cpu_adjoint_and_fd(rsd, ctx):
    g = golden("transient_adjoint_q1_hex_6x5x4.npz")
    h = make(rsd, ctx)
    dt, N = float(g["dt"]), int(g["nsteps"])
    theta, U0 = ctx.to_device(g["theta"]), ctx.to_device(g["U0"])
    U = ctx.array(h.n)
    rep = h.transient_forward(theta, U0, U, 0.0, dt, N, **TIGHT)
    assert rep["converged"]
    assert relerr(U.download(), g["UN"]) <= 1e-11
    dJdU = ctx.to_device(U.download() - g["Uobs"])
    grad = ctx.array(g["theta"].size)
    rep = h.transient_backward(theta, U0, dJdU, grad, 0.0, dt, N, **TIGHT)
    assert rep["converged"]
    C = math.ceil(math.sqrt(N))
    assert rep["states_held"] == math.ceil(N / C) + C + 1 < N + 1
    gd = grad.download()
    assert relerr(gd, g["grad"]) <= 1e-9
    assert abs(gd @ g["fd_dir"] - g["fd"]) <= 1e-6 * abs(g["fd"])

    # central differences through the device forward steps along 20 directions
    th = g["theta"]
    rs = np.random.default_rng(3)
    hstep = 1e-6
    Ut = ctx.array(h.n)

    def J(t):
        h.transient_forward(ctx.to_device(t), U0, Ut, 0.0, dt, N, **TIGHT)
        return 0.5 * float(np.sum((Ut.download() - g["Uobs"]) ** 2))
    errs = []
    for _ in range(20):
        d = rs.standard_normal(th.size)
        d /= np.linalg.norm(d)
        fd = (J(th + hstep * d) - J(th - hstep * d)) / (2 * hstep)
        errs.append(abs(fd - gd @ d) / abs(fd))
    assert max(errs) <= 1e-6, errs


def test_transient_autograd_function(rsd, ctx):
    torch = pytest.importorskip("torch")
    from importlib import import_module
    ag = import_module("residuum_solver_b200.autograd")
    g = golden("transient_adjoint_q1_hex_6x5x4.npz")
    h = make(rsd, ctx)
    theta = torch.tensor(g["theta"], dtype=torch.float64, device="cuda", requires_grad=True)
    U0 = torch.tensor(g["U0"], dtype=torch.float64, device="cuda")
    Uobs = torch.tensor(g["Uobs"], dtype=torch.float64, device="cuda")
    cfg = rsd.SolverConfig.make(**TIGHT)
    U = ag.HeatTransient.apply(theta, h, U0, 0.0, float(g["dt"]), int(g["nsteps"]), cfg)
    J = 0.5 * ((U - Uobs) ** 2).sum()
    J.backward()
    assert abs(J.item() - float(g["J"])) <= 1e-11 * abs(float(g["J"]))
    assert relerr(theta.grad.cpu().numpy(), g["grad"]) <= 1e-9


def test_transient_pair_edge_cases(rsd, ctx):
    g = golden("transient_adjoint_q1_hex_6x5x4.npz")
    h = make(rsd, ctx)
    theta, U0 = ctx.to_device(g["theta"]), ctx.to_device(g["U0"])
    grad = ctx.array(g["theta"].size).fill(1.0)
    dJdU = ctx.array(h.n).fill(1.0)
    rep = h.transient_backward(theta, U0, dJdU, grad, 0.0, 0.01, 0, **TIGHT)   # no steps: zero gradient
    assert rep["converged"] and not np.any(grad.download())
    with pytest.raises(rsd.RsdError):
        h.transient_backward(theta, U0, dJdU, grad, 0.0, -0.01, 3, **TIGHT)
    # one step: the steady-like gradient of a single Backward-Euler solve
    U = ctx.array(h.n)
    h.transient_forward(theta, U0, U, 0.0, 0.01, 1, **TIGHT)
    rep = h.transient_backward(theta, U0, dJdU, grad, 0.0, 0.01, 1, **TIGHT)
    assert rep["converged"] and rep["states_held"] == 3
