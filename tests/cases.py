"""Constructor arguments for the test structures (DDAModel argument names)."""
import math

import numpy as np


def model_args(nx, ny, nz, sici, *, d=25.0, lam=542.0, material=(1.0 + 0j, 3.5 + 0.01j), nback=1.0,
               MAXm=0, MAXn=0, Lm=None, Ln=None, method="FCD", symmetry="None", symaxis=(0.0, 0.0),
               seed=0, rho=None, geometry=None, n_K=(0, 0, 1), n_E0=(1, 0, 0), power=2.0):
    """Box (or given) geometry, x fastest; z-uniform column densities rho ~ U[0,1]
    drawn from `seed` unless `rho` (per dipole) is given."""
    from oracle.dda_oracle import generate_geometry

    if geometry is None:
        geometry = generate_geometry(nx, ny, nz)
    g = np.asarray(geometry).reshape(-1, 3)
    N = len(g)
    if rho is None:
        rng = np.random.default_rng(seed)
        col = rng.random((nx, ny))
        rho = col[g[:, 0], g[:, 1]]
    diel = np.repeat(np.asarray(rho, dtype=np.float64), 3)
    si, ci = sici
    return dict(
        betaMin=0.0, betaMax=50.0, ita=0.5, betaType="piecewise", filterIterations=[100],
        filterRadii=[2.0], useFilter=False, symmetryType=symmetry, symmetryAxis=list(symaxis),
        isPeriodic=MAXm > 0 or MAXn > 0, objectiveName="IntegratedE",
        objPara=[power, 0.0, nx - 1.0, 0.0, ny - 1.0, 0.0, nz - 1.0, 0.95, 50.0],
        geometry=np.asarray(geometry).ravel(), inputDielectrics=diel, num_x=nx, num_y=ny, num_z=nz,
        num_total=N, n_K=list(n_K), E0=1.0, n_E0=list(n_E0), lam=lam, material=list(material),
        nback=nback, MAXm=MAXm, MAXn=MAXn, Lm=nx if Lm is None else Lm, Ln=ny if Ln is None else Ln,
        matrixAMethodName=method, d=d, sineIntegralValues=si, cosineIntegralValues=ci,
        integralDelta=0.1, verbose=False)


def fixture22_args(fx, sici):
    """The reference's 22x22x10 test model (python_tests/test_DDAModel.py:8-104)."""
    nx, ny, nz, n = (int(v) for v in fx["header"])
    rho = np.unpackbits(fx["rho_bits"])[:n].astype(np.float64)
    si, ci = sici
    return dict(
        betaMin=0.0, betaMax=50.0, ita=0.5, betaType="piecewise", filterIterations=[100],
        filterRadii=[2.0], useFilter=False, symmetryType="4fold", symmetryAxis=[10.5, 10.5],
        isPeriodic=True, objectiveName="IntegratedE",
        objPara=[2.0, 0.0, 21.0, 0.0, 21.0, 0.0, 9.0, 0.95, 50.0],
        geometry=fx["geometry"].astype(np.int64), inputDielectrics=np.repeat(rho, 3),
        num_x=nx, num_y=ny, num_z=nz, num_total=n, n_K=[0, 0, 1], E0=1.0, n_E0=[1, 0, 0],
        lam=542.0, material=[1.01 + 0j, 5.96282 + 3.80423e-7j], nback=math.sqrt(1.01),
        MAXm=50, MAXn=50, Lm=22, Ln=22, matrixAMethodName="FCD", d=15.0,
        sineIntegralValues=si, cosineIntegralValues=ci, integralDelta=0.1, verbose=False)


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
