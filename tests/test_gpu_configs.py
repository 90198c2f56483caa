"""Full-size checks of the differentiation workload: 96x96x24
dipoles (221,184), periodic with period 96 d in x and y and the lattice sums
over |m|,|n| <= 50, raw design rho ~ U[0, 1] -> radius-2 cone filter -> tanh
projection (beta 8, eta 0.5), objective mean |E|^2 over an 8x8x1 patch 3
cells above the top face.  The structure fills its periodic cell, where
BiCGSTAB stalls; the solves use the deflated restarted GMRES solver in mixed
precision, refined to a 1e-11 true residual.

Tolerances: central differences with step 1e-5 of solves at a 1e-11 residual
carry ~1e-11 / 1e-5 of the objective as error; they are checked at 2e-3 of
the largest gradient entry plus 2% of the entry.  The finite-difference
solves start from the unperturbed solution (the perturbation is tiny)."""
import numpy as np
import pytest

from cases import model_args

pytestmark = pytest.mark.gpu

NX, NY, NZ = 96, 96, 24
M = 50
TOL = 1e-11
SOLVER = dict(degree=1, restart=100, deflate=30)


def _model(sici, rho=None, symmetry="None"):
    from dda_model import DDAModel

    kw = model_args(NX, NY, NZ, sici, MAXm=M, MAXn=M, rho=rho, symmetry=symmetry)
    m = DDAModel(**kw, precision="mixed")
    m.setSolver("pgmres", **SOLVER)
    return m


def _patch():
    c0x, c0y = NX // 2 - 4, NY // 2 - 4
    return np.array([[x, y, NZ - 1 + 3] for x in range(c0x, c0x + 8) for y in range(c0y, c0y + 8)])


def test_differentiation_workload_adjoint_vs_central_differences(sici):
    import torch

    from dda_model.autograd import design_densities, design_objective

    m = _model(sici)
    m.setObservationPoints(_patch())
    x0 = np.random.default_rng(44).random((NX, NY, NZ))
    x = torch.tensor(x0, dtype=torch.float64, device="cuda", requires_grad=True)
    J = design_objective(x, m, radius=2.0, beta=8.0, eta=0.5, kind="patch", tol=TOL)
    assert m.last_solve["status"] == "converged", m.last_solve
    P0 = m.getPolarization()
    J.backward()
    g = x.grad.cpu().numpy()
    assert m.last_adjoint["status"] == "converged", m.last_adjoint
    gmax = np.abs(g).max()
    assert np.isfinite(g).all() and gmax > 0
    stream = torch.cuda.current_stream().cuda_stream

    def Jx(a):
        with torch.no_grad():
            rho = design_densities(torch.tensor(a, device="cuda"), 2.0, 8.0, 0.5)
            m.setDensitiesDevice(rho.data_ptr(), stream)
            m.solveElectricField(P0, 400000, TOL)
            assert m.last_solve["status"] == "converged", m.last_solve
            return m.patchObjective()

    rng = np.random.default_rng(45)
    idx = [tuple(int(v) for v in (rng.integers(NX), rng.integers(NY), rng.integers(NZ))) for _ in range(20)]
    h = 1e-5
    for i in idx:
        e = np.zeros_like(x0)
        e[i] = h
        fd = (Jx(x0 + e) - Jx(x0 - e)) / (2 * h)
        assert abs(fd - g[i]) <= 2e-3 * gmax + 2e-2 * abs(g[i]), (i, fd, g[i], gmax)


def test_reference_gradient_algorithm_matches_exact_adjoint_at_full_size(sici):
    """calculateGradients (the reference's one-sided FD partials + adjoint
    solve, src/DDAModel.cpp:398-578) on z-extruded column parameters agrees
    with the exact adjoint gradient summed over each column, on the periodic
    structure."""
    rng = np.random.default_rng(46)
    col = rng.uniform(0.1, 0.9, (NX, NY))
    from oracle.dda_oracle import generate_geometry

    g3 = generate_geometry(NX, NY, NZ).reshape(-1, 3)
    rho = col[g3[:, 0], g3[:, 1]]
    m = _model(sici, rho=rho)
    m.solveElectricField(None, 400000, TOL)
    assert m.last_solve["status"] == "converged", m.last_solve
    J0 = m.calculateObjective()
    exact = m.gradientDensities(400000, TOL)
    per_col = np.zeros((NX, NY))
    np.add.at(per_col, (g3[:, 0], g3[:, 1]), exact)
    m.solveElectricField(None, 400000, TOL)
    ref = m.calculateGradients(1e-4, J0, 400000, TOL)
    # parameter k is the column of the first dipole carrying it (x fastest)
    ref_cols = ref.reshape(NY, NX).T
    scale = np.abs(per_col).max()
    assert np.abs(ref_cols - per_col).max() <= 5e-3 * scale
