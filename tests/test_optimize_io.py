"""Host-side parts of the optimisation driver and the file formats (no GPU):
penalty gradients against central differences, the coefficient schedules and
Adam against their defining formulas, and file round trips in the
reference's layouts."""
import math
import os

import numpy as np
import pytest


@pytest.mark.parametrize("kind,cfg", [("parabolic", {}), ("gaussian", {"sigma": 0.15, "mu": 0.5}),
                                      ("triangular", {"slope": 2.0})])
def test_penalty_gradients_match_central_differences(kind, cfg):
    from dda_model.optimize import penalty, penalty_gradient

    x = np.array([0.05, 0.2, 0.37, 0.61, 0.8, 0.97])
    h = 1e-6
    fd = (penalty(kind, x + h, cfg) - penalty(kind, x - h, cfg)) / (2 * h)
    assert np.allclose(fd, penalty_gradient(kind, x, cfg), rtol=1e-6, atol=1e-8)


def test_coefficient_schedules():
    from dda_model.optimize import coefficient

    pw = {"frac1": 0.25, "frac2": 0.5, "frac3": 0.75, "iter_end": 100, "coeff1": 0.0, "coeff2": 0.1,
          "coeff3": 0.2, "coeff4": 0.3}
    assert [coefficient("piecewise", i, pw) for i in (0, 25, 26, 50, 51, 75, 76, 99)] == \
        [0.0, 0.0, 0.1, 0.1, 0.2, 0.2, 0.3, 0.3]
    pa = {"iter1": 10, "iter2": 20, "iter3": 30, "coeff1": 1, "coeff2": 2, "coeff3": 3, "coeff4": 4}
    assert [coefficient("piecewise_absolute", i, pa) for i in (10, 11, 20, 21, 31)] == [1, 2, 2, 3, 4]
    lin = {"iter_start": 10, "iter_end": 50, "coeff_min": 0.1, "coeff_max": 0.5}
    assert coefficient("linear", 5, lin) == 0.1 and coefficient("linear", 60, lin) == 0.5
    assert coefficient("linear", 20, lin) == pytest.approx(0.1 + 0.4 * 20 / 50)
    ex = dict(lin, base=10.0)
    assert coefficient("exp", 30, ex) == pytest.approx(0.1 + 0.4 * (10 ** 0.5 - 1) / 9)
    assert coefficient("constant", 7, {"coeff_const": 0.25}) == 0.25


def test_adam_steps():
    from dda_model.optimize import Adam

    rng = np.random.default_rng(0)
    gs = [rng.standard_normal(5) for _ in range(4)]
    opt = Adam()
    V = S = 0.0
    for t, g in enumerate(gs):
        V = 0.9 * V + (1 - 0.9) * g / (1 - 0.9 ** (t + 1))
        S = 0.99 * S + (1 - 0.99) * g * g / (1 - 0.99 ** (t + 1))
        assert np.allclose(opt(g), V / (np.sqrt(S) + 1e-8), rtol=1e-14, atol=0)
    # the first step is the sign of the gradient
    assert np.allclose(Adam()(gs[0]), np.sign(gs[0]), rtol=1e-6)


def test_geometry_and_dielectric_files_round_trip(tmp_path, fixture22):
    from dda_model import io

    nx, ny, nz, n = (int(v) for v in fixture22["header"])
    geo = fixture22["geometry"].astype(np.int64)
    io.write_geometry(tmp_path / "geometry.txt", nx, ny, nz, geo)
    lines = open(tmp_path / "geometry.txt").read().split()
    assert lines[:4] == [str(nx), str(ny), str(nz), str(n)] and len(lines) == 4 + 3 * n
    gx = io.read_geometry(tmp_path / "geometry.txt")
    assert gx[:4] == (nx, ny, nz, n) and np.array_equal(gx[4], geo)
    rho = np.repeat(np.unpackbits(fixture22["rho_bits"])[:n].astype(np.float64), 3)
    io.write_dielectrics(tmp_path / "dielectrics.txt", rho)
    assert np.array_equal(io.read_dielectrics(tmp_path / "dielectrics.txt", n), rho)
    with pytest.raises(ValueError):
        io.read_dielectrics(tmp_path / "dielectrics.txt", n + 1)


def test_run_outputs_layout(tmp_path):
    from dda_model import io
    from dda_model.optimize import History

    io.create_output_directories(tmp_path)
    io.save_iteration(tmp_path, 3, structure=np.arange(6.0), e_field=np.array([1 + 2j, 3 - 1j]),
                      params=np.ones(2), penalty=np.zeros(2), penalty_gradient=np.ones(2))
    h = History(objective=[1.0, 2.0], coefficient=[0.0, 0.1], average_penalty=[0.2, 0.1], step_size=[0.01, 0.01])
    io.save_summary(tmp_path, h, "parabolic", {})
    for f in ("Structures/Structure3.txt", "E-Fields/E-Field3.txt", "Parameters/Param3.txt",
              "Penalties/Penalty3.txt", "Gradient_Penalties/Gradient3.txt", "Obj.txt", "Coeffs.txt",
              "Average_Penalties.txt", "stepsizes.txt", "Penalty_Shape.txt", "PenaltyGradient_Shape.txt"):
        assert os.path.exists(tmp_path / f), f
    assert np.allclose(np.loadtxt(tmp_path / "Obj.txt"), [1.0, 2.0])
    assert np.loadtxt(tmp_path / "Penalty_Shape.txt", delimiter=",").shape == (200, 2)
    assert np.allclose(np.loadtxt(tmp_path / "E-Fields/E-Field3.txt", dtype=complex), [1 + 2j, 3 - 1j])
