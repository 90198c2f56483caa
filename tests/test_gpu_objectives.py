"""Observation-patch objective, per-dipole density gradients and the torch
autograd bridge: CUDA path (through the C ABI) vs the oracle's dense direct
forward/adjoint solves and vs central finite differences.

Tolerances: solves run to a 1e-12 residual, so fields and gradients agree with
the dense direct solution to 1e-9 relative (the complex128 parity bar);
finite differences of objectives solved to 1e-12 at step 1e-5 carry ~1e-7
relative error, checked at 1e-5 of the largest gradient entry."""
import numpy as np
import pytest

from cases import model_args, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _pair(kw):
    from dda_model import DDAModel
    from oracle.dda_oracle import OracleModel

    return DDAModel(**kw), OracleModel(**kw)


def _obs(nx, ny, nz):
    # above the slab, below it, and beside it (outside the period cell)
    return np.array([[1, 2, nz + 2], [nx - 1, 0, nz + 1], [2, 3, -2], [-3, 2, 1], [nx + 2, ny + 1, nz + 4]])


@pytest.mark.parametrize("periodic,method", [(0, "FCD"), (1, "FCD"), (2, "LDR")])
def test_observation_field_matches_oracle(sici, periodic, method):
    kw = model_args(6, 5, 3, sici, MAXm=periodic, MAXn=periodic, method=method, seed=21)
    dev, ora = _pair(kw)
    obs = _obs(6, 5, 3)
    dev.solveElectricField(np.zeros(3 * ora.N, complex), 100000, TOL)
    ora.P = np.linalg.solve(ora.dense_operator(), ora.E)
    dev.setObservationPoints(obs)
    e_dev = dev.observationField()
    e_ora = ora.observation_field(obs).ravel()
    assert e_dev.shape == (3 * len(obs),)
    assert rel(e_dev, e_ora) < 1e-9
    assert abs(dev.patchObjective() / ora.patch_objective(obs) - 1) < 1e-9


def test_observation_points_inside_the_box(sici):
    """Empty cells of a non-box structure are valid observation points; a
    point on a dipole is rejected."""
    from dda_model import TddaError
    from oracle.dda_oracle import generate_geometry

    g = generate_geometry(6, 6, 3).reshape(-1, 3)
    keep = ~((g[:, 0] >= 2) & (g[:, 0] <= 3) & (g[:, 1] >= 2) & (g[:, 1] <= 3))  # a hole
    kw = model_args(6, 6, 3, sici, MAXm=1, MAXn=1, geometry=g[keep], seed=4)
    dev, ora = _pair(kw)
    dev.solveElectricField(np.zeros(3 * ora.N, complex), 100000, TOL)
    ora.P = np.linalg.solve(ora.dense_operator(), ora.E)
    obs = np.array([[2, 2, 1], [3, 2, 0], [2, 3, 5]])
    dev.setObservationPoints(obs)
    assert rel(dev.observationField(), ora.observation_field(obs).ravel()) < 1e-9
    with pytest.raises(TddaError):
        dev.setObservationPoints(np.array([[0, 0, 0]]))


@pytest.mark.parametrize("kind", ["integrated", "patch"])
@pytest.mark.parametrize("periodic", [0, 1])
def test_density_gradient_matches_oracle(sici, kind, periodic):
    kw = model_args(6, 5, 3, sici, MAXm=periodic, MAXn=periodic, seed=22)
    dev, ora = _pair(kw)
    rho = np.random.default_rng(23).uniform(0.0, 1.0, ora.N)
    dev.setDensities(rho)
    ora.set_densities(rho)
    assert np.array_equal(dev.getDielectrics(), ora.getDielectrics())
    obs = _obs(6, 5, 3)
    dev.solveElectricField(np.zeros(3 * ora.N, complex), 100000, TOL)
    if kind == "integrated":
        g_dev = dev.gradientDensities(100000, TOL)
    else:
        dev.setObservationPoints(obs)
        g_dev = dev.patchGradient(100000, TOL)
    assert dev.last_adjoint["status"] == "converged"
    g_ora = ora.density_gradient(kind, obs)
    assert g_dev.shape == (ora.N,)
    assert rel(g_dev, g_ora) < 1e-9


@pytest.mark.parametrize("kind", ["integrated", "patch"])
def test_density_gradient_matches_central_differences(sici, kind):
    from dda_model import DDAModel

    kw = model_args(5, 5, 2, sici, MAXm=1, MAXn=1, seed=24)
    dev = DDAModel(**kw)
    obs = _obs(5, 5, 2)
    dev.setObservationPoints(obs)
    rho = np.random.default_rng(25).uniform(0.05, 0.95, dev.N)

    def J(r):
        dev.setDensities(r)
        dev.solveElectricField(None, 100000, TOL)
        return dev.calculateObjective() if kind == "integrated" else dev.patchObjective()

    J(rho)
    g = dev.gradientDensities(100000, TOL) if kind == "integrated" else dev.patchGradient(100000, TOL)
    h = 1e-5
    for j in (0, 7, dev.N - 1):
        e = np.zeros(dev.N)
        e[j] = h
        fd = (J(rho + e) - J(rho - e)) / (2 * h)
        assert abs(fd - g[j]) <= 1e-5 * np.abs(g).max()


@pytest.mark.parametrize("kind", ["integrated", "patch"])
def test_autograd_design_chain(sici, kind):
    """d J(project(filter(x))) / dx through torch autograd and the CUDA adjoint,
    against central differences of the whole chain."""
    import torch

    from dda_model import DDAModel
    from dda_model.autograd import design_objective

    nx, ny, nz = 6, 6, 3
    kw = model_args(nx, ny, nz, sici, MAXm=1, MAXn=1, seed=26)
    dev = DDAModel(**kw)
    dev.setObservationPoints(_obs(nx, ny, nz))
    x0 = np.random.default_rng(27).uniform(0.2, 0.8, (nx, ny, nz))
    x = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
    J = design_objective(x, dev, radius=1.5, beta=4.0, kind=kind, tol=TOL)
    J.backward()
    g = x.grad.numpy()
    assert np.isfinite(g).all() and np.abs(g).max() > 0

    def Jx(a):
        with torch.no_grad():
            return float(design_objective(torch.tensor(a), dev, radius=1.5, beta=4.0, kind=kind, tol=TOL))

    h = 1e-5
    for idx in [(0, 0, 0), (2, 3, 1), (5, 4, 2)]:
        e = np.zeros_like(x0)
        e[idx] = h
        fd = (Jx(x0 + e) - Jx(x0 - e)) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * np.abs(g).max()
