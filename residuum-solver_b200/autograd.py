"""torch.autograd.Functions over the adjoint pairs rsd_heat_forward / rsd_heat_backward (steady)
and rsd_heat_transient_forward / rsd_heat_transient_backward (Backward-Euler steps).

    T = HeatSolve.apply(theta, heat, cfg)      # theta: CUDA float64 tensor, one value per element
    J = 0.5 * ((T - T_obs) ** 2).sum(); J.backward()   # theta.grad = dJ/dtheta by the adjoint

    U_N = HeatTransient.apply(theta, heat, U0, t0, dt, nsteps, cfg)   # the state after nsteps steps

The library runs on its own stream and returns when its results are complete; the wrapper makes
that stream wait for torch's work on the inputs by synchronizing torch's current stream first.
"""
import torch

from . import SolverConfig


class HeatSolve(torch.autograd.Function):
    @staticmethod
    def forward(fctx, theta, heat, cfg=None):
        cfg = cfg or SolverConfig.make(tol=1e-12, max_iters=100000)
        theta = theta.detach().contiguous()
        T = torch.zeros(heat.n, dtype=torch.float64, device=theta.device)
        torch.cuda.current_stream(theta.device).synchronize()
        heat.forward(theta, T, cfg)
        fctx.heat, fctx.cfg = heat, cfg
        fctx.save_for_backward(theta, T)
        return T

    @staticmethod
    def backward(fctx, grad_T):
        theta, T = fctx.saved_tensors
        g = torch.empty_like(theta)
        grad_T = grad_T.contiguous()
        torch.cuda.current_stream(theta.device).synchronize()
        fctx.heat.backward(theta, T, grad_T, g, fctx.cfg)
        return g, None, None


class HeatTransient(torch.autograd.Function):
    """U_N after nsteps Backward-Euler steps from U0; backward replays the steps from checkpoints
    (nothing but theta and U0 is saved) and returns dJ/dtheta."""

    @staticmethod
    def forward(fctx, theta, heat, U0, t0, dt, nsteps, cfg=None):
        cfg = cfg or SolverConfig.make(tol=1e-12, max_iters=100000)
        theta = theta.detach().contiguous()
        U0 = U0.detach().contiguous()
        U = torch.empty_like(U0)
        torch.cuda.current_stream(theta.device).synchronize()
        heat.transient_forward(theta, U0, U, t0, dt, nsteps, cfg)
        fctx.heat, fctx.cfg, fctx.args = heat, cfg, (t0, dt, nsteps)
        fctx.save_for_backward(theta, U0)
        return U

    @staticmethod
    def backward(fctx, grad_U):
        theta, U0 = fctx.saved_tensors
        g = torch.empty_like(theta)
        grad_U = grad_U.contiguous()
        torch.cuda.current_stream(theta.device).synchronize()
        t0, dt, nsteps = fctx.args
        fctx.heat.transient_backward(theta, U0, grad_U, g, t0, dt, nsteps, fctx.cfg)
        return g, None, None, None, None, None, None
