"""Topology-optimisation driver over DDAModel.

The loop of calculation_scripts/TopoOptCalculation.py:165-209: objective,
objective gradient, binarisation penalty and its gradient with a scheduled
coefficient, Adam, a clipped ascent step on the free parameters.  Two
differences make it cheaper on the GPU:

* gradient="adjoint" (default) takes the exact gradient -- one adjoint solve
  with the same operator, d(1/alpha)/drho in closed form, summed over each
  parameter's dipoles -- instead of the reference's one-sided finite
  differences (gradient="reference" keeps those, src/DDAModel.cpp:398-578);
* warm_start=True starts every forward solve from the previous iteration's
  polarisation (the design moves little per step), where the reference starts
  from zero.

Adam, the penalties and the coefficient schedules follow
python_bindings/dda_model/optimizers.py:3-23 and binarizers.py:5-93 formula
for formula (they define the optimisation trajectory).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import io as dio


# --- binarisation penalties (binarizers.py:5-34) ------------------------------
def penalty(kind, x, cfg):
    x = np.asarray(x, dtype=np.float64)
    if kind == "parabolic":
        return x - x * x
    if kind == "gaussian":
        sig, mu = cfg["sigma"], cfg["mu"]
        return sig * np.exp(-np.square((x - mu) / sig) / 2 + 0.5)
    if kind == "triangular":
        s = cfg["slope"]
        return np.where(x > 0.5, s - s * x, s * x)
    raise ValueError(f"unknown penalty {kind!r}")


def penalty_gradient(kind, x, cfg):
    x = np.asarray(x, dtype=np.float64)
    if kind == "parabolic":
        return 1 - 2 * x
    if kind == "gaussian":
        sig, mu = cfg["sigma"], cfg["mu"]
        return -(x - mu) * penalty("gaussian", x, cfg) / (sig * sig)
    if kind == "triangular":
        s = cfg["slope"]
        return np.where(x > 0.5, -s, s) * np.ones_like(x)
    raise ValueError(f"unknown penalty {kind!r}")


# --- penalty coefficient schedules (binarizers.py:36-93) ----------------------
def coefficient(kind, it, cfg):
    if kind == "constant":
        return cfg["coeff_const"]
    if kind == "piecewise_absolute":
        bounds = (cfg["iter1"], cfg["iter2"], cfg["iter3"])
        coeffs = (cfg["coeff1"], cfg["coeff2"], cfg["coeff3"], cfg["coeff4"])
        for b, c in zip(bounds, coeffs):
            if it <= b:
                return c
        return coeffs[3]
    if kind == "piecewise":
        end = cfg["iter_end"]
        bounds = (cfg["frac1"] * end, cfg["frac2"] * end, cfg["frac3"] * end)
        coeffs = (cfg["coeff1"], cfg["coeff2"], cfg["coeff3"], cfg["coeff4"])
        for b, c in zip(bounds, coeffs):
            if it <= b:
                return c
        return coeffs[3]
    if kind in ("linear", "exp"):
        start, end = cfg["iter_start"], cfg["iter_end"]
        lo, hi = cfg["coeff_min"], cfg["coeff_max"]
        if it < start:
            return lo
        if it > end:
            return hi
        if kind == "linear":
            return lo + (hi - lo) * it / end
        base = cfg["base"]
        return lo + (hi - lo) * (math.pow(base, (it - start) / (end - start)) - 1) / (base - 1)
    raise ValueError(f"unknown coefficient schedule {kind!r}")


class Adam:
    """optimizers.py:3-23, including its bias correction inside the moving
    averages: V <- b1 V + (1 - b1) g / (1 - b1^(t+1)),
    S <- b2 S + (1 - b2) g^2 / (1 - b2^(t+1)), step = V / (sqrt(S) + 1e-8)."""

    def __init__(self, beta1=0.9, beta2=0.99):
        self.beta1, self.beta2 = beta1, beta2
        self.V = 0.0
        self.S = 0.0
        self.timestep = 0

    def __call__(self, g):
        g = np.asarray(g, dtype=np.float64)
        t = self.timestep
        self.V = self.beta1 * self.V + (1 - self.beta1) * g / (1 - self.beta1 ** (t + 1))
        self.S = self.beta2 * self.S + (1 - self.beta2) * g * g / (1 - self.beta2 ** (t + 1))
        self.timestep += 1
        return self.V / (np.sqrt(self.S) + 1e-8)


@dataclass
class History:
    objective: list = field(default_factory=list)
    coefficient: list = field(default_factory=list)
    average_penalty: list = field(default_factory=list)
    step_size: list = field(default_factory=list)
    iterations: list = field(default_factory=list)   # BiCGSTAB iterations of each forward solve


class TopologyOptimization:
    """Gradient ascent of the IntegratedE objective of `model` (a DDAModel)
    over its free parameters.  data_path (optional) receives the reference's
    per-iteration files (Structures/, Parameters/, Penalties/,
    Gradient_Penalties/, E-Fields/ and the summary files)."""

    def __init__(self, model, step_size=0.01, penalty_type="parabolic", penalty_config=None,
                 coeff_type="constant", coeff_config=None, optimizer=None, gradient="adjoint",
                 warm_start=True, bgs_max_iter=100_000, bgs_max_error=1e-5, fd_epsilon=1e-3, data_path=None):
        if gradient not in ("adjoint", "reference"):
            raise ValueError("gradient must be 'adjoint' or 'reference'")
        self.m = model
        self.step_size = step_size
        self.penalty_type = penalty_type
        self.penalty_config = penalty_config or {}
        self.coeff_type = coeff_type
        self.coeff_config = coeff_config if coeff_config is not None else {"coeff_const": 0.0}
        self.opt = optimizer or Adam()
        self.gradient = gradient
        self.warm_start = warm_start
        self.max_iter, self.tol, self.fd_eps = bgs_max_iter, bgs_max_error, fd_epsilon
        self.data_path = data_path
        self.history = History()
        self._P = None
        self._map = model.parameterMap() if gradient == "adjoint" else None
        if data_path:
            dio.create_output_directories(data_path)

    def objective(self):
        P0 = self._P if (self.warm_start and self._P is not None) else np.zeros(3 * self.m.N, complex)
        self.m.solveElectricField(P0, self.max_iter, self.tol)
        self.history.iterations.append(self.m.last_solve["iterations"])
        if self.warm_start:
            self._P = self.m.getPolarization()
        return self.m.calculateObjective()

    def objective_gradient(self, J):
        if self.gradient == "reference":
            return self.m.calculateGradients(self.fd_eps, J, self.max_iter, self.tol)
        g = self.m.gradientDensities(self.max_iter, self.tol)
        return np.bincount(self._map, weights=g, minlength=self.m.NFpara)

    def step(self, it):
        """One iteration of TopoOptCalculation.py:165-209."""
        h = self.history
        J = self.objective()
        h.objective.append(J)
        g_obj = self.objective_gradient(J)
        params = self.m.getParameters()
        if self.data_path:
            dio.save_iteration(self.data_path, it, structure=self.m.getDielectrics(),
                               e_field=self.m.getElectricField(), params=params)
        pg = penalty_gradient(self.penalty_type, params, self.penalty_config)
        pen = penalty(self.penalty_type, params, self.penalty_config)
        if self.data_path:
            dio.save_iteration(self.data_path, it, penalty=pen, penalty_gradient=pg)
        h.average_penalty.append(float(np.average(pen)))
        coeff = coefficient(self.coeff_type, it, self.coeff_config)
        h.coefficient.append(coeff)
        grads = (1 - coeff) * g_obj - coeff * pg
        h.step_size.append(self.step_size)
        new = np.clip(params + self.step_size * self.opt(grads), 0, 1)
        self.m.setParameters(new)
        return J

    def run(self, iterations):
        for it in range(iterations):
            self.step(it)
        if self.data_path:
            dio.save_summary(self.data_path, self.history, self.penalty_type, self.penalty_config)
        return self.history
