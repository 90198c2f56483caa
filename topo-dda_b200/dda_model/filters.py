"""Design-density chain: radius-R cone filter and tanh projection.

These replace the reference's in-plane cone filter + exponential projection
(src/DDAModel.cpp:580-712, src/FilterOption.cpp:48-62), which every Python
path of the reference disables, with the 3-D form the benchmark configurations
use:

* cone filter of radius R (in cells): rho~_i = sum_j w_ij rho_j / sum_j w_ij,
  w_ij = max(0, R - |r_i - r_j|); periodic in x and y (the structure is a
  period of an infinite lattice), truncated and renormalised in z;
* tanh projection: (tanh(beta eta) + tanh(beta (x - eta))) /
  (tanh(beta eta) + tanh(beta (1 - eta))).

Arrays are indexed [x, y, z].  Both numpy and torch inputs are accepted; the
torch path is differentiable (autograd).
"""
from __future__ import annotations

import itertools
import math

import numpy as np


def cone_offsets(radius: float):
    """Integer offsets with positive cone weight and their weights."""
    r = int(math.ceil(radius))
    offs, ws = [], []
    for dx, dy, dz in itertools.product(range(-r, r + 1), repeat=3):
        w = radius - math.sqrt(dx * dx + dy * dy + dz * dz)
        if w > 0:
            offs.append((dx, dy, dz))
            ws.append(w)
    return offs, np.asarray(ws)


def _shift_z(a, dz, lib):
    """a shifted by dz along z (axis 2) with zero fill (no wrap)."""
    nz = a.shape[2]
    if dz == 0:
        return a
    out = lib.zeros_like(a)
    if abs(dz) >= nz:
        return out
    if dz > 0:
        out[:, :, dz:] = a[:, :, :nz - dz]
    else:
        out[:, :, :nz + dz] = a[:, :, -dz:]
    return out


def cone_filter(rho, radius: float = 2.0):
    """Cone filter of the given radius (cells); rho indexed [x, y, z]."""
    try:
        import torch

        is_t = isinstance(rho, torch.Tensor)
    except ImportError:  # pragma: no cover
        is_t = False
    lib = __import__("torch") if is_t else np
    offs, ws = cone_offsets(radius)
    ones = lib.ones_like(rho)
    num = lib.zeros_like(rho)
    den = lib.zeros_like(rho)
    for (dx, dy, dz), w in zip(offs, ws):
        if is_t:
            sh = lib.roll(rho, shifts=(dx, dy), dims=(0, 1))
            sh1 = lib.roll(ones, shifts=(dx, dy), dims=(0, 1))
        else:
            sh = np.roll(rho, shift=(dx, dy), axis=(0, 1))
            sh1 = np.roll(ones, shift=(dx, dy), axis=(0, 1))
        num = num + float(w) * _shift_z(sh, dz, lib)
        den = den + float(w) * _shift_z(sh1, dz, lib)
    return num / den


def tanh_projection(x, beta: float = 8.0, eta: float = 0.5):
    try:
        import torch

        if isinstance(x, torch.Tensor):
            t = torch.tanh
            return (math.tanh(beta * eta) + t(beta * (x - eta))) / (
                math.tanh(beta * eta) + math.tanh(beta * (1 - eta)))
    except ImportError:  # pragma: no cover
        pass
    return (np.tanh(beta * eta) + np.tanh(beta * (x - eta))) / (
        np.tanh(beta * eta) + np.tanh(beta * (1 - eta)))


def binary_design(nx: int, ny: int, nz: int, seed: int, fill: float = 0.5):
    """Seeded binary 0/1 field indexed [x, y, z]."""
    rng = np.random.default_rng(seed)
    return (rng.random((nx, ny, nz)) < fill).astype(np.float64)


def dipole_order(field_xyz: np.ndarray) -> np.ndarray:
    """[x, y, z] array -> per-dipole vector in the x-fastest geometry order."""
    return np.ascontiguousarray(np.transpose(field_xyz, (2, 1, 0)).ravel())
