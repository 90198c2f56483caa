"""Differentiable DDA objectives for torch.

`dda_objective(rho, model)` runs the forward solve for per-dipole densities
`rho` (a torch tensor) and returns the objective; its backward pass is the
hand-written adjoint of libtdda (one adjoint solve with the same,
complex-symmetric operator -- src/DDAModel.cpp:429-435 -- then d(1/alpha)/drho
in closed form), not finite differences.  `design_objective` prepends the
radius-R cone filter and the tanh projection, run by libtdda's design kernels
with their hand-written adjoints, so the gradient reaches the raw design field.
CUDA tensors stay on the device from the raw design to the gradient: the
library reads the densities and writes the gradient through device pointers,
on the current CUDA stream.

Objectives: "integrated" -- the reference's IntegratedE, log sum |al P|^q
(src/ObjDDAModel.cpp:103-218); "patch" -- mean |E|^2 over the observation
points set with model.setObservationPoints.
"""
from __future__ import annotations

import torch

from . import _lib


def _stream():
    return torch.cuda.current_stream().cuda_stream


class _Design(torch.autograd.Function):
    """raw[x, y, z] -> cone filter -> tanh projection -> densities (dipole order)."""

    @staticmethod
    def forward(ctx, raw, radius, beta, eta):
        raw = raw.detach().to(torch.float64).contiguous()
        nx, ny, nz = raw.shape
        filtered = torch.empty_like(raw)
        rho = torch.empty(nx * ny * nz, dtype=torch.float64, device=raw.device)
        _lib.check(_lib.load().tdda_design_forward_device(nx, ny, nz, float(radius), float(beta), float(eta),
                                                          raw.data_ptr(), filtered.data_ptr(), rho.data_ptr(),
                                                          _stream()))
        ctx.save_for_backward(filtered)
        ctx.args = (nx, ny, nz, float(radius), float(beta), float(eta))
        return rho

    @staticmethod
    def backward(ctx, g_rho):
        (filtered,) = ctx.saved_tensors
        nx, ny, nz, radius, beta, eta = ctx.args
        g_rho = g_rho.to(torch.float64).contiguous()
        g_raw = torch.empty_like(filtered)
        scratch = torch.empty_like(filtered)
        _lib.check(_lib.load().tdda_design_backward_device(nx, ny, nz, radius, beta, eta, filtered.data_ptr(),
                                                           g_rho.data_ptr(), g_raw.data_ptr(), scratch.data_ptr(),
                                                           _stream()))
        return g_raw, None, None, None


class _DDAObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, model, kind, max_iter, tol):
        if kind not in ("integrated", "patch"):
            raise ValueError("kind must be 'integrated' or 'patch'")
        r = rho.detach().to(torch.float64).contiguous()
        if r.is_cuda:
            model.setDensitiesDevice(r.data_ptr(), _stream())
        else:
            model.setDensities(r.numpy())
        model.solveElectricField(None, max_iter, tol)
        J = model.calculateObjective() if kind == "integrated" else model.patchObjective()
        ctx.model, ctx.kind, ctx.max_iter, ctx.tol = model, kind, max_iter, tol
        ctx.device, ctx.dtype = rho.device, rho.dtype
        return torch.tensor(J, dtype=rho.dtype, device=rho.device)

    @staticmethod
    def backward(ctx, grad_out):
        m = ctx.model
        if ctx.device.type == "cuda":
            g = torch.empty(m.N, dtype=torch.float64, device=ctx.device)
            fn = m.gradientDensitiesDevice if ctx.kind == "integrated" else m.patchGradientDevice
            fn(g.data_ptr(), ctx.max_iter, ctx.tol, _stream())
        else:
            g = torch.from_numpy(m.gradientDensities(ctx.max_iter, ctx.tol) if ctx.kind == "integrated"
                                 else m.patchGradient(ctx.max_iter, ctx.tol))
        return grad_out * g.to(ctx.dtype), None, None, None, None


def dda_objective(rho, model, kind="patch", max_iter=100000, tol=1e-10):
    """Objective of the structure with per-dipole densities rho (dipole order)."""
    return _DDAObjective.apply(rho, model, kind, max_iter, tol)


def design_densities(rho_xyz, radius=2.0, beta=8.0, eta=0.5):
    """rho_xyz[x, y, z] -> cone filter (radius in cells) -> tanh projection ->
    densities in dipole order (x fastest), computed on the GPU (differentiable;
    a CPU tensor is moved to the GPU and its gradient flows back)."""
    dev = rho_xyz if rho_xyz.is_cuda else rho_xyz.to("cuda")
    return _Design.apply(dev.to(torch.float64), radius, beta, eta)


def design_objective(rho_xyz, model, radius=2.0, beta=8.0, eta=0.5, kind="patch", max_iter=100000,
                     tol=1e-10):
    """rho_xyz[x, y, z] -> cone filter (radius in cells) -> tanh projection ->
    densities in dipole order (x fastest) -> objective."""
    return dda_objective(design_densities(rho_xyz, radius, beta, eta), model, kind, max_iter, tol)
