"""Internal consistency of the oracle: table quirks, lattice symmetry, FFT
convolution vs a dense operator, BiCGSTAB vs a direct solve, adjoint vs
finite differences."""
import math

import numpy as np
import pytest

from cases import model_args, rel


def test_sici_lookup_quirks(sici):
    from oracle import dda_oracle as O

    lib = O._load_lib()
    si, ci = sici
    dp = O._dptr
    # interpolation between entries k and k+1, read as if at (k+1)*delta
    x = 12.34
    k = int(math.floor(x / 0.1)) - 1
    expect = si[k] + (si[k + 1] - si[k]) / (((k + 2) * 0.1) - ((k + 1) * 0.1)) * (x - (k + 1) * 0.1)
    assert lib.oracle_get_si(dp(si), len(si), 0.1, x) == pytest.approx(expect, rel=1e-15)
    # beyond the table: last entry
    assert lib.oracle_get_ci(dp(ci), len(ci), 0.1, 1e7) == ci[-1]
    # exact multiple of delta: the table value (the reference would give NaN)
    before = lib.oracle_guard_hits()
    v = lib.oracle_get_si(dp(si), len(si), 0.1, 0.5)
    assert np.isfinite(v) and v == si[4]
    assert lib.oracle_guard_hits() == before + 1


@pytest.mark.parametrize("method", ["FCD", "LDR"])
def test_octant_lattice_equals_full_evaluation(sici, method):
    from oracle import dda_oracle as O

    si, ci = sici
    K = 2 * math.pi / 542.0
    kw = dict(Nx=5, Ny=4, Nz=3, d=25.0, K=K, Lm=5 * 25.0, Ln=4 * 25.0, MAXm=3, MAXn=2, method=method,
              si=si, ci=ci, delta=0.1)
    a = O.lattice_tensor(**kw, full=False)
    b = O.lattice_tensor(**kw, full=True)
    assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))
    # without periodic images the zero offset is the (zero) self term
    kw.update(MAXm=0, MAXn=0)
    assert np.all(O.lattice_tensor(**kw)[0, 0, 0] == 0)


@pytest.mark.parametrize("periodic", [False, True])
def test_fft_aproduct_matches_dense_operator(sici, periodic):
    from oracle.dda_oracle import OracleModel

    kw = model_args(4, 3, 2, sici, MAXm=2 if periodic else 0, MAXn=1 if periodic else 0, seed=3)
    m = OracleModel(**kw)
    M = m.dense_operator()
    rng = np.random.default_rng(1)
    x = rng.standard_normal(3 * m.N) + 1j * rng.standard_normal(3 * m.N)
    assert rel(m.aproduct_with_alb(x), M @ x) < 1e-13
    # complex symmetric (the adjoint reuses the forward operator)
    assert np.max(np.abs(M - M.T)) <= 1e-14 * np.max(np.abs(M))


def test_bicgstab_matches_direct_solve(sici):
    from oracle.dda_oracle import OracleModel

    m = OracleModel(**model_args(5, 4, 3, sici, seed=5))
    m.solveElectricField(np.zeros(3 * m.N, complex), 1000, 1e-13)
    direct = np.linalg.solve(m.dense_operator(), m.E)
    assert rel(m.P, direct) < 1e-11
    assert m.last_info.converged


def test_reference_gradient_close_to_analytic_adjoint(sici):
    """The reference's one-sided FD partials agree with the exact adjoint
    gradient to O(eps)."""
    from oracle.dda_oracle import OracleModel, bicgstab

    m = OracleModel(**model_args(4, 4, 2, sici, seed=7))
    m.solveElectricField(np.zeros(3 * m.N, complex), 1000, 1e-13)
    J = m.calculateObjective()
    P = m.P.copy()
    al = m.al.copy()
    S = m.E_int
    # exact: dJ/drho_i = explicit - Re(lambda^T (dal o P)), A lambda = 2 |al|^2 conj(P) / S
    devp = 2 * np.abs(al) ** 2 * np.conj(P) / S
    lam, _ = bicgstab(m.aproduct_with_alb, devp, np.zeros_like(devp), 1000, 1e-13)
    dal = np.repeat(m.dal_drho(), 3)
    explicit = (2 * np.real(np.conj(al) * dal) * np.abs(P) ** 2 / S).reshape(-1, 3).sum(1)
    per_dipole = explicit - np.real((lam * dal * P).reshape(-1, 3).sum(1))
    exact = np.zeros(m.NFpara)
    np.add.at(exact, m.geometryPara, per_dipole)
    fd = m.calculateGradients(1e-4, J, 1000, 1e-13)
    # one-sided differences are O(eps) accurate where 1/alpha(rho) is smooth;
    # near rho = 0 (vacuum) it is steep and the reference's partials degrade
    base = m.getParameters()
    ok = base > 0.05
    assert ok.sum() >= 10
    assert rel(fd[ok], exact[ok]) < 5e-3
    # central differences of J confirm the exact gradient, including near rho = 0
    h = 1e-5
    for k in (3, int(np.argmin(base))):
        vals = []
        for s in (+1, -1):
            v = base.copy()
            v[k] += s * h
            m.setParameters(v)
            m.solveElectricField(np.zeros(3 * m.N, complex), 1000, 1e-13)
            vals.append(m.calculateObjective())
        assert (vals[0] - vals[1]) / (2 * h) == pytest.approx(exact[k], rel=1e-5)


@pytest.mark.parametrize("kind", ["integrated", "patch"])
def test_density_gradient_matches_central_differences(sici, kind):
    """The oracle's dense exact-adjoint density gradient (the checker of the
    CUDA adjoint) against central differences of the directly solved objective."""
    from oracle.dda_oracle import OracleModel

    m = OracleModel(**model_args(4, 4, 2, sici, MAXm=1, MAXn=1, seed=11))
    obs = np.array([[x, y, 4] for x in (1, 2) for y in (1, 3)])
    rho = np.random.default_rng(12).uniform(0.1, 0.9, m.N)

    def J(r):
        m.set_densities(r)
        m.P = np.linalg.solve(m.dense_operator(), m.E)
        if kind == "integrated":
            return m.calculateObjective()
        return m.patch_objective(obs)

    m.set_densities(rho)
    g = m.density_gradient(kind, obs)
    assert g.shape == (m.N,)
    h = 1e-6
    for j in (0, 5, m.N - 1):
        e = np.zeros(m.N)
        e[j] = h
        fd = (J(rho + e) - J(rho - e)) / (2 * h)
        assert abs(fd - g[j]) <= 1e-6 * np.abs(g).max()
