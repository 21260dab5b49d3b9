"""Differentiable scattering intensities: adjoint solve behind torch.autograd.

The reference has no derivatives; this module adds them on top of the same
operator (``multiscat_gmres.f90:452-687``).  For intensities I = |S|^2 from

    A(V) psi = u,    S_G = 2i b_G psi_G(z_n) + delta_{G,spec} a_spec,

and a real loss L(I), one extra solve A^H lambda = -i gamma conj(b) e_n with
gamma_G = 2 (dL/dI_G) S_G gives dL/dV_d(z) = -2 conj(sum_G conj(lambda_G(z))
psi_{G-d}(z)) (only Re V_0 enters, so dL/dV_0 is real).  The forward psi stays
on the device between forward and backward; the adjoint solve reuses the
forward plan (eigenbasis, tuning, graphs) with the operator switched to A^H.
"""

from __future__ import annotations

import numpy as np
import torch

from .solver import ScatteringPlan, SystemSpec


class _ScatteringIntensities(torch.autograd.Function):
    @staticmethod
    def forward(ctx, potential: torch.Tensor, kinetic, systems, plan_kwargs, window):
        v = potential.detach().to("cpu", torch.complex128).numpy()
        plan = ScatteringPlan(v, kinetic, systems, **plan_kwargs)
        res = plan.solve()
        ctx.plan = plan
        ctx.window = window
        ctx.device = potential.device
        ctx.save_for_backward(res.psi)
        return res.intensities.to(potential.device)

    @staticmethod
    def backward(ctx, grad_intensities):
        (psi,) = ctx.saved_tensors
        plan: ScatteringPlan = ctx.plan
        g = grad_intensities.to(psi.device, torch.float64).contiguous()
        lam = plan.solve_adjoint(psi, dl_dintensity=g).psi
        grad_v = plan.potential_gradient(psi, lam, ctx.window)
        return grad_v.to(ctx.device), None, None, None, None


def scattering_intensities(potential: torch.Tensor, kinetic, systems: list[SystemSpec], *,
                           window: tuple[int, int] | None = None, **plan_kwargs) -> torch.Tensor:
    """|S_G|^2 of every channel row of every system (float64 [total_rows], on
    the GPU), differentiable with respect to ``potential`` (complex128
    [nkx, nky, nz], natural units).  ``window`` = (half_x, half_y) limits the
    gradient to offsets |dx| <= half_x, |dy| <= half_y (others get 0);
    ``plan_kwargs`` go to :class:`ScatteringPlan` (rtol, precision, ...)."""
    return _ScatteringIntensities.apply(potential, np.asarray(kinetic, float), systems,
                                        dict(plan_kwargs), window)


def weighted_intensity_loss(potential: torch.Tensor, kinetic, systems: list[SystemSpec],
                            weights: torch.Tensor, **plan_kwargs) -> torch.Tensor:
    """L = sum_rows w_row |S_row|^2 (weights float64 [total_rows])."""
    inten = scattering_intensities(potential, kinetic, systems, **plan_kwargs)
    return (weights.to(inten.device, torch.float64) * inten).sum()
