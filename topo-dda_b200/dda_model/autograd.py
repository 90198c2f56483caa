"""Differentiable DDA objectives for torch.

`dda_objective(rho, model)` runs the forward solve for per-dipole densities
`rho` (a torch tensor) and returns the objective; its backward pass is the
hand-written adjoint of libtdda (one adjoint solve with the same,
complex-symmetric operator -- src/DDAModel.cpp:429-435 -- then d(1/alpha)/drho
in closed form), not finite differences.  `design_objective` prepends the
radius-R cone filter and the tanh projection (dda_model.filters) in torch, so
autograd carries the gradient back to the raw design field.

Objectives: "integrated" -- the reference's IntegratedE, log sum |al P|^q
(src/ObjDDAModel.cpp:103-218); "patch" -- mean |E|^2 over the observation
points set with model.setObservationPoints.
"""
from __future__ import annotations

import torch

from . import filters


class _DDAObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, model, kind, max_iter, tol):
        model.setDensities(rho.detach().to("cpu", torch.float64).numpy())
        model.solveElectricField(None, max_iter, tol)
        if kind == "integrated":
            J = model.calculateObjective()
        elif kind == "patch":
            J = model.patchObjective()
        else:
            raise ValueError("kind must be 'integrated' or 'patch'")
        ctx.model, ctx.kind, ctx.max_iter, ctx.tol = model, kind, max_iter, tol
        ctx.device, ctx.dtype = rho.device, rho.dtype
        return torch.tensor(J, dtype=rho.dtype, device=rho.device)

    @staticmethod
    def backward(ctx, grad_out):
        m = ctx.model
        if ctx.kind == "integrated":
            g = m.gradientDensities(ctx.max_iter, ctx.tol)
        else:
            g = m.patchGradient(ctx.max_iter, ctx.tol)
        return grad_out * torch.from_numpy(g).to(ctx.device, ctx.dtype), None, None, None, None


def dda_objective(rho, model, kind="patch", max_iter=100000, tol=1e-10):
    """Objective of the structure with per-dipole densities rho (dipole order)."""
    return _DDAObjective.apply(rho, model, kind, max_iter, tol)


def design_objective(rho_xyz, model, radius=2.0, beta=8.0, eta=0.5, kind="patch", max_iter=100000,
                     tol=1e-10):
    """rho_xyz[x, y, z] -> cone filter (radius in cells) -> tanh projection ->
    densities in dipole order (x fastest) -> objective."""
    f = filters.cone_filter(rho_xyz, radius)
    p = filters.tanh_projection(f, beta, eta).clamp(0.0, 1.0)
    dip = p.permute(2, 1, 0).reshape(-1)
    return dda_objective(dip, model, kind, max_iter, tol)
