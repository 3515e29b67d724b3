"""torch.autograd over the render: film = render(theta) with theta the field parameters
(plane-wave amplitudes and phases, or spline coefficients), and d/dtheta from the adjoint kernel.

    theta = torch.tensor(simpler_b200.field_params(setup), requires_grad=True)
    film = RenderFunction.apply(theta, setup, n_photons)          # (Z, Y, X) float64, CPU
    loss = (film * roi).sum(); loss.backward()                   # theta.grad = dloss/dtheta

The forward pass renders with the given parameters; the backward pass calls the adjoint with
dJ/dfilm = the incoming gradient, on the same photons and Philox seed, so the gradient is the
pathwise derivative of the very estimator the forward pass returned.
"""
from __future__ import annotations

import numpy as np
import torch

from ..render import adjoint, render, with_field_params


class RenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, setup, n_photons: int) -> torch.Tensor:
        s = with_field_params(setup, theta.detach().cpu().numpy())
        film, _ = render(s, int(n_photons))
        ctx.setup = s
        ctx.n_photons = int(n_photons)
        return torch.from_numpy(film)

    @staticmethod
    def backward(ctx, grad_film: torch.Tensor):
        g = np.ascontiguousarray(grad_film.detach().cpu().numpy(), dtype=np.float64)
        grad, _ = adjoint(ctx.setup, ctx.n_photons, g)
        return torch.from_numpy(grad), None, None


def render_torch(theta: torch.Tensor, setup, n_photons: int) -> torch.Tensor:
    """film = render(setup with field parameters theta), differentiable in theta."""
    return RenderFunction.apply(theta, setup, n_photons)
