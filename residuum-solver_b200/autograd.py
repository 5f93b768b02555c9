"""torch.autograd.Function over the adjoint pair rsd_heat_forward / rsd_heat_backward.

    T = HeatSolve.apply(theta, heat, cfg)      # theta: CUDA float64 tensor, one value per element
    J = 0.5 * ((T - T_obs) ** 2).sum(); J.backward()   # theta.grad = dJ/dtheta by the adjoint

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
