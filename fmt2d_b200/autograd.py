"""The traveltime misfit as a differentiable PyTorch function of the
propagation-grid slowness.

forward: the model's velocity becomes 1/slowness (fmt2d_update_model), the
time fields of the sources are solved (fmt2d_forward) and the picks traced;
the value is 0.5 * sum(((t_calc - t_obs) / sigma)^2) over the valid picks.
backward: the discrete adjoint of the time fields (fmt2d_misfit_gradient)
gives the misfit's exact derivative with respect to every grid node's
slowness, computed with the forward and kept for the backward call.

The reference has no such gradient: its inversion builds the ray-based
Frechet rows (compute_frechet_for_ray2d, src/inversion2d.f90:4548-4787) and
forms G^T r inside LSQR; that is what fmt2d_trace / fmt2d_frechet_rows
return and what the adjoint gradient is compared against.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native


class EikonalMisfit(torch.autograd.Function):
    """misfit = EikonalMisfit.apply(slowness, g, src_x, phases, picks, t_obs,
    sigma): slowness a (nz, nx) tensor on any device, g an api.Fmt2d holding
    the model (its numbering is kept: the slowness only changes the
    velocities), picks a dict of arrays src, phase, rx, rz (phases 1-3)."""

    @staticmethod
    def forward(ctx, slowness, g, src_x, phases, picks, t_obs, sigma):
        s = slowness.detach().to("cpu", torch.float64).numpy()
        if s.shape != (g.nz, g.nx):
            raise ValueError(f"slowness must be ({g.nz}, {g.nx}), got {tuple(s.shape)}")
        if not np.all(s > 0.0):
            raise ValueError("slowness must be positive")
        g.update_model(vel=1.0 / s)
        g.forward(src_x, phases)
        out = g.misfit_gradient(picks["src"], picks["phase"], picks["rx"], picks["rz"], t_obs,
                                sigma)
        bad = out["info"][:3]
        if np.any(bad != 0):
            raise _native.Fmt2dError(f"adjoint could not follow the forward: {bad.tolist()}")
        grad = torch.from_numpy(out["grad_slow"]).to(slowness.device, slowness.dtype)
        ctx.save_for_backward(grad)
        ctx.extra = {"t_calc": out["t_calc"], "valid": out["valid"]}
        return torch.tensor(out["misfit"], dtype=torch.float64, device=slowness.device)

    @staticmethod
    def backward(ctx, gout):
        (grad,) = ctx.saved_tensors
        return (gout.to(grad.dtype) * grad, None, None, None, None, None, None)


def eikonal_misfit(slowness, g, src_x, phases, picks, t_obs, sigma):
    """The misfit as a differentiable function of slowness (EikonalMisfit)."""
    return EikonalMisfit.apply(slowness, g, src_x, phases, picks, t_obs, sigma)
