"""dda_model — B200-native drop-in for Topo-DDA's `dda_model` package.

Exports the same names as python_bindings/dda_model/__init__.py:
``DDAModel`` (the pybind11 class, here over the libtdda C ABI),
``DDAModelWrapper`` and ``_generate_geometry``.
"""
from __future__ import annotations

import numpy as np

from ._dda_model import DDAModel
from ._lib import TddaError

__all__ = ["DDAModel", "DDAModelWrapper", "TddaError", "_generate_geometry", "sici_tables"]


def _generate_geometry(num_x: int, num_y: int, num_z: int) -> np.ndarray:
    """Integer voxel coordinates, x fastest, flattened as [x0, y0, z0, x1, ...]
    (python_bindings/dda_model/__init__.py:8-20)."""
    z, y, x = np.meshgrid(np.arange(num_z), np.arange(num_y), np.arange(num_x), indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).ravel().astype(int)


def sici_tables(delta: float = 0.1, n: int = 1_000_000):
    """Sine/cosine-integral tables in the layout the FCD kernel looks up:
    n-1 samples of linspace(delta, delta*n, n-1), read as if at (k+1)*delta
    (python_bindings/dda_model/__init__.py:205-210, src/SiCi.cpp:12-44)."""
    from scipy.special import sici

    return sici(np.linspace(delta, delta * n, n - 1))


class DDAModelWrapper:
    """Keyword-friendly construction of a DDAModel with the reference defaults
    (FCD, MAXm = MAXn = 50, 4-fold symmetry, periodic; filter disabled) —
    python_bindings/dda_model/__init__.py:23-203.  ``precision`` selects the
    complex128 path (default) or mixed precision."""

    def __init__(self, num_pixels_xyz, pixel_size_nm, initial_parameter_values, dielectric_constants,
                 light_direction, light_polarization, light_wavelength_nm, light_amplitude=1.0,
                 symmetry_axes=(), symmetry_method="4fold", symmetry_is_periodic=True,
                 integral_power=2, integral_xbounds=None, integral_ybounds=None, integral_zbounds=None,
                 background_refractive_index=None, objective_name="IntegratedE", apc_max_m=50,
                 apc_max_n=50, apc_l_m=None, apc_l_n=None, apc_method_name="FCD", verbose=False,
                 precision="complex128"):
        if len(num_pixels_xyz) != 3:
            raise ValueError("num_pixels_xyz must contain the number of pixels in [x, y, z] but "
                             f"instead found {num_pixels_xyz}.")
        if len(symmetry_axes) != 2 and symmetry_method == "4fold":
            raise ValueError("If symmetry_method is 4fold, symmetry_axes must be 2-dimensional. "
                             f"Instead found {symmetry_axes}.")
        self._pixel_dimensions = list(num_pixels_xyz)
        nx, ny, nz = (int(v) for v in num_pixels_xyz)
        ntot = nx * ny * nz
        geometry = _generate_geometry(nx, ny, nz)
        xb = list(integral_xbounds) if integral_xbounds else [0.0, float(nx) - 1]
        yb = list(integral_ybounds) if integral_ybounds else [0.0, float(ny) - 1]
        zb = list(integral_zbounds) if integral_zbounds else [0.0, float(nz) - 1]
        objective_config = [integral_power] + xb + yb + zb + [0.95, 50.0]
        l_n = apc_l_n if apc_l_n else nx
        l_m = apc_l_m if apc_l_m else ny
        si, ci = sici_tables(0.1, 1_000_000)
        nback = background_refractive_index
        if not nback:
            nback = float(np.sqrt(np.real(dielectric_constants[0])))
        self._model = DDAModel(
            0.0, 50.0, 0.5, "piecewise", [100], [2.0], False,
            symmetry_method, list(symmetry_axes), symmetry_is_periodic,
            objective_name, objective_config,
            geometry, initial_parameter_values,
            nx, ny, nz, ntot,
            light_direction, light_amplitude, light_polarization,
            light_wavelength_nm, dielectric_constants, nback,
            apc_max_m, apc_max_n, l_m, l_n, apc_method_name, pixel_size_nm,
            si, ci, 0.1, verbose, precision=precision)

    def objective(self, bgs_max_iter: int = 100_000, bgs_max_error: float = 1e-5):
        n = int(np.prod(self._pixel_dimensions))
        self._model.solveElectricField(np.zeros(3 * n, dtype=np.complex128), bgs_max_iter, bgs_max_error)
        return self._model.calculateObjective()

    def gradients(self, current_objective_value: float, finite_difference_epsilon: float = 0.001,
                  bgs_max_iter: int = 100_000, bgs_max_error: float = 1e-5):
        return self._model.calculateGradients(finite_difference_epsilon, current_objective_value,
                                              bgs_max_iter, bgs_max_error)

    @property
    def parameters(self):
        return self._model.getParameters()

    @parameters.setter
    def parameters(self, value):
        self._model.setParameters(value)

    def allParameters(self):
        return self._model.getDielectrics()

    def getElectricField(self):
        return self._model.getElectricField()
