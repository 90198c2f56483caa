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

import ctypes
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


_PENALTY_KIND = {"parabolic": 0, "gaussian": 1, "triangular": 2}


class DeviceTopologyOptimization(TopologyOptimization):
    """The same loop with its state on the GPU: the free parameters, Adam's
    moving averages, the per-dipole and per-parameter gradients and the
    penalties live in device memory.  Per iteration: parameters -> densities
    through the parameter map, a forward solve warm-started from the model's
    own polarisation, the objective (computed by the solve's last kernel), the
    exact adjoint gradient into device memory, its per-parameter sums, and the
    update (penalty, penalised gradient, Adam, clipped step) in one kernel --
    only scalars (objective, coefficient, mean penalty) reach the host.  Each
    operation is rounded as the host loop rounds it, so both follow the same
    trajectory.  The exact adjoint gradient only (gradient="adjoint");
    data_path files are written from device copies.  The model's parameters
    are set from the device state when run() ends."""

    def __init__(self, model, *args, device="cuda", **kwargs):
        super().__init__(model, *args, **kwargs)
        if self.gradient != "adjoint":
            raise ValueError("the device loop takes the exact adjoint gradient")
        if not isinstance(self.opt, Adam):
            raise ValueError("the device loop runs the reference's Adam")
        if self.penalty_type not in _PENALTY_KIND:
            raise ValueError(f"unknown penalty {self.penalty_type!r}")
        import torch

        self._torch = torch
        f64 = dict(dtype=torch.float64, device=device)
        self.params = torch.from_numpy(model.getParameters()).to(**f64)
        self.V = torch.zeros_like(self.params)
        self.S = torch.zeros_like(self.params)
        self.g_obj = torch.zeros_like(self.params)
        self.pen = torch.zeros_like(self.params)
        self.pen_grad = torch.zeros_like(self.params)
        self.pen_mean = torch.zeros(1, **f64)
        self.rho = torch.zeros(model.N, **f64)
        self.g_rho = torch.zeros(model.N, **f64)
        self._first = True

    def step(self, it):
        from . import _lib

        torch, m, h = self._torch, self.m, self.history
        stream = torch.cuda.current_stream().cuda_stream
        m.paramsToDensitiesDevice(self.params.data_ptr(), self.rho.data_ptr(), stream)
        m.setDensitiesDevice(self.rho.data_ptr(), stream)
        if self._first or not self.warm_start:
            m.solveElectricField(None, self.max_iter, self.tol)
            self._first = False
        else:
            m.solveElectricFieldWarm(self.max_iter, self.tol)
        h.iterations.append(m.last_solve["iterations"])
        J = m.calculateObjective()
        h.objective.append(J)
        m.gradientDensitiesDevice(self.g_rho.data_ptr(), self.max_iter, self.tol, stream)
        m.densitiesToParamsDevice(self.g_rho.data_ptr(), self.g_obj.data_ptr(), stream)
        if self.data_path:
            dio.save_iteration(self.data_path, it, structure=m.getDielectrics(), e_field=m.getElectricField(),
                               params=self.params.cpu().numpy())
        coeff = coefficient(self.coeff_type, it, self.coeff_config)
        h.coefficient.append(coeff)
        a = self.opt
        t = a.timestep
        cfg = self.penalty_config
        c = _lib.AscentStep(penalty=_PENALTY_KIND[self.penalty_type], sigma=float(cfg.get("sigma", 1.0)),
                            mu=float(cfg.get("mu", 0.5)), slope=float(cfg.get("slope", 1.0)), coeff=float(coeff),
                            one_minus_coeff=float(1 - coeff), step=float(self.step_size), beta1=a.beta1,
                            beta2=a.beta2, one_minus_beta1=1 - a.beta1, one_minus_beta2=1 - a.beta2,
                            bias1=1 - a.beta1 ** (t + 1), bias2=1 - a.beta2 ** (t + 1))
        a.timestep += 1
        _lib.check(_lib.load().tdda_ascent_step_device(
            self.params.numel(), self.params.data_ptr(), self.V.data_ptr(), self.S.data_ptr(),
            self.g_obj.data_ptr(), ctypes.byref(c), self.pen.data_ptr(), self.pen_grad.data_ptr(),
            self.pen_mean.data_ptr(), stream))
        if self.data_path:
            dio.save_iteration(self.data_path, it, penalty=self.pen.cpu().numpy(),
                               penalty_gradient=self.pen_grad.cpu().numpy())
        h.average_penalty.append(float(self.pen_mean.item()))
        h.step_size.append(self.step_size)
        return J

    def run(self, iterations):
        hist = super().run(iterations)
        self.m.setParameters(self.params.cpu().numpy())
        return hist
