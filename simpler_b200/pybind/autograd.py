"""torch.autograd over the render: film = render(theta) with theta the field parameters (Bessel
amplitude and phase window, plane-wave amplitudes and phases, or spline coefficients), and
d/dtheta from the adjoint kernels.

    theta = torch.tensor(simpler_b200.field_params(setup), requires_grad=True)
    film = render_torch(theta, setup, n_photons)                 # (Z, Y, X) float64 on cuda:device
    loss = (film * roi).sum(); loss.backward()                   # theta.grad = dloss/dtheta

The forward pass renders into a resident plan and copies the film device to device into a CUDA
tensor (no host round trip); the backward pass hands the incoming gradient to the same plan's
adjoint (photons [0, n_photons), the same Philox seed), so the gradient is the pathwise derivative
of the very estimator the forward pass returned. A plan is kept per (setup, parameters) for the
autograd graph's life.
"""
from __future__ import annotations

import numpy as np
import torch

from ..render import Plan, with_field_params


class RenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, setup, n_photons: int) -> torch.Tensor:
        s = with_field_params(setup, theta.detach().cpu().numpy())
        plan = Plan(s)
        n = int(n_photons)
        device = torch.device("cuda", s.device)
        stream = torch.cuda.current_stream(device).cuda_stream
        plan.clear(stream)
        plan.trace(0, n, n, stream)
        film = torch.empty(s.film_shape(), dtype=torch.float64, device=device)
        plan.read_image_device(film.data_ptr(), stream)
        ctx.plan = plan
        ctx.n_photons = n
        ctx.theta_device = theta.device
        return film

    @staticmethod
    def backward(ctx, grad_film: torch.Tensor):
        g = np.ascontiguousarray(grad_film.detach().cpu().numpy(), dtype=np.float64)
        grad, _ = ctx.plan.adjoint(g, 0, ctx.n_photons, ctx.n_photons)
        ctx.plan.close()
        return torch.from_numpy(grad).to(ctx.theta_device), None, None


def render_torch(theta: torch.Tensor, setup, n_photons: int) -> torch.Tensor:
    """film = render(setup with field parameters theta), differentiable in theta; a CUDA tensor."""
    return RenderFunction.apply(theta, setup, n_photons)
