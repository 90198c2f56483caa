"""The reference's file formats.

Inputs (python_tests/data): ``geometry.txt`` -- num_x, num_y, num_z,
num_total, then 3 * num_total voxel coordinates, one integer per line;
``dielectrics.txt`` -- 3 * num_total densities, one per line.

Outputs of an optimisation run, as calculation_scripts/TopoOptCalculation.py
writes them under <run>/Data (read back by its plotScript.py): one value per
line, per iteration ``Structures/Structure{i}.txt`` (every dipole's density,
3 per dipole), ``Parameters/Param{i}.txt``, ``Penalties/Penalty{i}.txt``,
``Gradient_Penalties/Gradient{i}.txt``, ``E-Fields/E-Field{i}.txt`` (complex
values as numpy writes them), and once ``Obj.txt``, ``Coeffs.txt``,
``Average_Penalties.txt``, ``stepsizes.txt`` and ``Penalty_Shape.txt`` /
``PenaltyGradient_Shape.txt`` (200 samples of x in [0, 1], "x,value").
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

OUTPUT_DIRS = ("Structures", "Parameters", "Penalties", "Gradient_Penalties", "E-Fields")


def read_geometry(path):
    """(num_x, num_y, num_z, num_total, geometry int[3 * num_total])."""
    v = np.loadtxt(path, dtype=np.int64).ravel()
    nx, ny, nz, n = (int(t) for t in v[:4])
    g = v[4:]
    if g.size != 3 * n:
        raise ValueError(f"{path}: header says {n} dipoles, found {g.size // 3}")
    return nx, ny, nz, n, g


def write_geometry(path, nx, ny, nz, geometry):
    g = np.asarray(geometry, dtype=np.int64).ravel()
    np.savetxt(path, np.concatenate([[nx, ny, nz, g.size // 3], g]), fmt="%d")


def read_dielectrics(path, num_total=None):
    d = np.loadtxt(path, dtype=np.float64).ravel()
    if num_total is not None and d.size != 3 * num_total:
        raise ValueError(f"{path}: expected {3 * num_total} values, found {d.size}")
    return d


def write_dielectrics(path, values):
    np.savetxt(path, np.asarray(values, dtype=np.float64).ravel(), delimiter="\n")


def create_output_directories(data_path):
    for d in OUTPUT_DIRS:
        Path(os.path.join(data_path, d)).mkdir(parents=True, exist_ok=True)


def save_iteration(data_path, it, structure=None, e_field=None, params=None, penalty=None, penalty_gradient=None):
    items = (("Structures", f"Structure{it}.txt", structure), ("E-Fields", f"E-Field{it}.txt", e_field),
             ("Parameters", f"Param{it}.txt", params), ("Penalties", f"Penalty{it}.txt", penalty),
             ("Gradient_Penalties", f"Gradient{it}.txt", penalty_gradient))
    for d, name, v in items:
        if v is not None:
            np.savetxt(os.path.join(data_path, d, name), np.asarray(v).ravel(), delimiter="\n")


def save_summary(data_path, history, penalty_type=None, penalty_config=None):
    for name, v in (("Obj.txt", history.objective), ("Coeffs.txt", history.coefficient),
                    ("Average_Penalties.txt", history.average_penalty), ("stepsizes.txt", history.step_size)):
        np.savetxt(os.path.join(data_path, name), np.asarray(v, dtype=np.float64), delimiter="\n")
    if penalty_type is not None:
        from .optimize import penalty, penalty_gradient

        x = np.linspace(0, 1, 200)
        np.savetxt(os.path.join(data_path, "Penalty_Shape.txt"),
                   np.column_stack((x, penalty(penalty_type, x, penalty_config))), delimiter=",")
        np.savetxt(os.path.join(data_path, "PenaltyGradient_Shape.txt"),
                   np.column_stack((x, penalty_gradient(penalty_type, x, penalty_config))), delimiter=",")
