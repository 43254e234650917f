"""The traveltime misfit as a differentiable PyTorch function of the
propagation-grid slowness and of the inverted interface's node depths.

forward: the model's velocity becomes 1/slowness and, when given, the
inverted interface (the Moho by default) takes the new node depths
(fmt2d_update_model); the time fields of the sources are solved
(fmt2d_forward) and the picks traced; the value is
0.5 * sum(((t_calc - t_obs) / sigma)^2) over the valid picks.
backward: the discrete adjoint of the time fields (fmt2d_misfit_gradient)
gives the misfit's exact derivative with respect to every grid node's
slowness and every interface node's depth, computed with the forward and
kept for the backward call.

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
    """misfit = EikonalMisfit.apply(slowness, iface_z, g, src_x, phases,
    picks, t_obs, sigma): slowness a (nz, nx) tensor on any device; iface_z
    None or an (nx,) tensor of the inverted interface's node depths; g an
    api.Fmt2d holding the model (its numbering must not change); picks a dict
    of arrays src, phase, rx, rz (phases 1-5)."""

    @staticmethod
    def forward(ctx, slowness, iface_z, g, src_x, phases, picks, t_obs, sigma):
        s = slowness.detach().to("cpu", torch.float64).numpy()
        if s.shape != (g.nz, g.nx):
            raise ValueError(f"slowness must be ({g.nz}, {g.nx}), got {tuple(s.shape)}")
        if not np.all(s > 0.0):
            raise ValueError("slowness must be positive")
        z = None
        if iface_z is not None:
            z = iface_z.detach().to("cpu", torch.float64).numpy()
            if z.shape != (g.nx,):
                raise ValueError(f"iface_z must be ({g.nx},), got {tuple(z.shape)}")
        g.update_model(vel=1.0 / s, iface_z=z)
        g.forward(src_x, phases)
        out = g.misfit_gradient(picks["src"], picks["phase"], picks["rx"], picks["rz"], t_obs,
                                sigma, want=("slow", "iface"))
        bad = out["info"][:3]
        if np.any(bad != 0):
            raise _native.Fmt2dError(f"adjoint could not follow the forward: {bad.tolist()}")
        gs = torch.from_numpy(out["grad_slow"]).to(slowness.device, slowness.dtype)
        if iface_z is not None:
            gz = torch.from_numpy(out["grad_iface"][g.iface_inv - 1].copy()).to(
                iface_z.device, iface_z.dtype)
        else:
            gz = torch.zeros(0)
        ctx.save_for_backward(gs, gz)
        ctx.has_z = iface_z is not None
        ctx.extra = {"t_calc": out["t_calc"], "valid": out["valid"]}
        return torch.tensor(out["misfit"], dtype=torch.float64, device=slowness.device)

    @staticmethod
    def backward(ctx, gout):
        gs, gz = ctx.saved_tensors
        dz = gout.to(gz.dtype) * gz if ctx.has_z else None
        return (gout.to(gs.dtype) * gs, dz, None, None, None, None, None, None)


def eikonal_misfit(slowness, g, src_x, phases, picks, t_obs, sigma, iface_z=None):
    """The misfit as a differentiable function of slowness and, when given,
    of the inverted interface's node depths (EikonalMisfit)."""
    return EikonalMisfit.apply(slowness, iface_z, g, src_x, phases, picks, t_obs, sigma)
