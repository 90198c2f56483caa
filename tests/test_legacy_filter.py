"""The reference's legacy design filter: the oracle's restatement on the CPU
(schedules, projection, weights), and the device implementation behind
DDAModel(useFilter=True) against it.

Tolerance: the device sums the weights in the reference's order with every
product and sum rounded separately; the projection's exp differs from the
host's by a few ulp, so parameters and gradients are checked at 1e-12
relative."""
import math

import numpy as np
import pytest

from cases import model_args


def test_beta_schedules_known_values():
    from oracle.dda_oracle import beta_schedule

    # piecewise (src/Tools.cpp:482-496): beta_min up to half, then 1/5, 1/2.5, then beta_max
    assert beta_schedule("piecewise", 50, 100, 0.0, 50.0) == 0.0
    assert beta_schedule("piecewise", 60, 100, 0.0, 50.0) == 10.0
    assert beta_schedule("piecewise", 75, 100, 0.0, 50.0) == 20.0
    assert beta_schedule("piecewise", 81, 100, 0.0, 50.0) == 50.0
    assert beta_schedule("linear", 25, 100, 10.0, 50.0) == 20.0
    assert beta_schedule("exp", 100, 100, 0.0, 99.0) == pytest.approx(99.0)
    assert beta_schedule("exp", 301, 400, 0.0, 99.0) == 0.5
    with pytest.raises(RuntimeError):
        beta_schedule("cubic", 1, 2, 0.0, 1.0)


def test_projection_is_continuous_and_monotone():
    from oracle.dda_oracle import smooth_density, smooth_density_d

    for beta in (0.5, 8.0, 50.0):
        for ita in (0.3, 0.5):
            a = smooth_density(ita, beta, ita)
            b = smooth_density(ita + 1e-12, beta, ita)
            assert abs(a - b) < 1e-9
            xs = np.linspace(0, 1, 101)
            v = [smooth_density(x, beta, ita) for x in xs]
            assert all(np.diff(v) >= -1e-15)
            assert smooth_density_d(0.2, beta, ita) > 0


def test_weights_are_the_in_plane_circle():
    from oracle.dda_oracle import LegacyFilter, generate_geometry, parameter_map

    g = generate_geometry(6, 5, 2)
    gp, p2g, nf = parameter_map(g, 2, "None", [0, 0])
    F = LegacyFilter(g, p2g, nf, 2.0, True, 6, 5, 0.0, 50.0, 0.5, "piecewise", np.full(nf, 0.5))
    # radius 2: the cell, 4 edge neighbours and 4 diagonal ones (d^2 <= 3.99)
    assert all(len(w) == 9 for w in F.weights)
    assert sorted(round(w, 12) for w, _ in F.weights[0]) == sorted(
        [2.0] + [1.0] * 4 + [round(2 - math.sqrt(2), 12)] * 4)
    F2 = LegacyFilter(g, p2g, nf, 2.0, False, 6, 5, 0.0, 50.0, 0.5, "piecewise", np.full(nf, 0.5))
    assert len(F2.weights[0]) == 4  # the corner cell without images


def _filter_model(sici, nx, ny, nz, periodic, symmetry, beta_type, radius, seed):
    kw = model_args(nx, ny, nz, sici, MAXm=1 if periodic else 0, MAXn=1 if periodic else 0, seed=seed,
                    symmetry=symmetry, symaxis=((nx - 1) / 2, (ny - 1) / 2))
    kw.update(useFilter=True, filterRadii=[radius], filterIterations=[100], betaType=beta_type,
              betaMin=1.0, betaMax=40.0, ita=0.5, isPeriodic=periodic)
    return kw


@pytest.mark.gpu
@pytest.mark.parametrize("periodic,symmetry,beta_type,radius", [(True, "None", "piecewise", 2.0),
                                                                (False, "None", "linear", 2.5),
                                                                (True, "4fold", "exp", 3.0)])
def test_device_filter_matches_oracle(sici, periodic, symmetry, beta_type, radius):
    from dda_model import DDAModel
    from oracle.dda_oracle import LegacyFilter, OracleModel

    nx, ny, nz = 10, 10, 3
    kw = _filter_model(sici, nx, ny, nz, periodic, symmetry, beta_type, radius, 5)
    dev = DDAModel(**kw)
    ora = OracleModel(**kw)
    F = LegacyFilter(ora.geometry, ora.p2g, ora.NFpara, radius, periodic, nx, ny, 1.0, 40.0, 0.5, beta_type,
                     ora.parameters)
    rng = np.random.default_rng(7)
    for it in (10, 60, 85):
        step = 0.3 * (rng.random(ora.NFpara) - 0.5)
        dev.updateStructure(step, it, 100)
        phys = F.update(step, it, 100)
        raw, filt, beta = dev.filterState()
        assert beta == F.beta
        assert np.array_equal(raw, F.origin)
        assert np.max(np.abs(filt - F.filtered)) <= 1e-15
        assert np.max(np.abs(dev.getParameters() - phys)) <= 1e-12
        ora.setParameters(phys)
        assert np.max(np.abs(dev.getDielectrics() - ora.getDielectrics())) <= 1e-12
        grad = rng.standard_normal(ora.NFpara)
        gd = dev.filterGradients(grad, it, 100)
        go = F.gradients(grad, it, 100)
        assert np.linalg.norm(gd - go) <= 1e-12 * np.linalg.norm(go)
    # the filtered structure solves like any other
    dev.solveElectricField(None, 10000, 1e-10)
    ora.solveElectricField(np.zeros(3 * ora.N, complex), 10000, 1e-10)
    assert np.linalg.norm(dev.getElectricField() - ora.EResult) <= 1e-8 * np.linalg.norm(ora.EResult)


@pytest.mark.gpu
def test_filter_entry_points_need_use_filter(sici):
    from dda_model import DDAModel
    from dda_model._lib import TddaError

    m = DDAModel(**model_args(6, 6, 2, sici))
    with pytest.raises(TddaError, match="useFilter"):
        m.updateStructure(np.zeros(m.NFpara), 1, 10)
