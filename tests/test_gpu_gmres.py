"""The polynomial-preconditioned GMRES solver (tdda_set_solver kind 1) vs the
oracle: the true residual of its solution, recomputed with the oracle's
complex128 operator, meets the tolerance, and the solution agrees with the
oracle's dense direct solve within the conditioning of the system
(1e3 x tol), in complex128 and in mixed precision, for periodic structures
that fill their cell (where the solver is meant to be used), non-box
geometries and several right-hand sides at once."""
import numpy as np
import pytest

from cases import model_args, rel

pytestmark = pytest.mark.gpu


def _solve(kw, precision, degree, restart, tol, B, max_iter=200000, deflate=0, kind="pgmres"):
    import torch

    from dda_model import DDAModel

    m = DDAModel(**kw, precision=precision)
    m.setSolver(kind, degree=degree, restart=restart, deflate=deflate)
    nrhs = B.shape[0]
    Bd = torch.from_numpy(B).cuda()
    X = torch.zeros_like(Bd)
    infos = m.solve_batch_device(Bd.data_ptr(), X.data_ptr(), nrhs, True, max_iter, tol,
                                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return X.cpu().numpy(), infos


def _rhs(ora, nrhs, seed):
    r = np.random.default_rng(seed)
    B = [ora.E]
    for _ in range(nrhs - 1):
        B.append(r.standard_normal(3 * ora.N) + 1j * r.standard_normal(3 * ora.N))
    return np.ascontiguousarray(np.stack(B))


@pytest.mark.parametrize("precision", ["complex128", "mixed"])
@pytest.mark.parametrize("shape,M,subset,nrhs", [((12, 12, 6), 20, False, 1), ((10, 8, 4), 5, True, 2),
                                                 ((16, 16, 8), 50, False, 1)])
def test_pgmres_matches_oracle(sici, precision, shape, M, subset, nrhs):
    from oracle.dda_oracle import OracleModel, generate_geometry

    nx, ny, nz = shape
    geo, rho = None, None
    if subset:
        # whole columns removed: the reference's parameter map needs N / Nz columns
        g = generate_geometry(nx, ny, nz).reshape(-1, 3)
        keep = (g[:, 0] * 3 + g[:, 1]) % 5 != 0
        geo = g[keep].ravel()
        rho = np.random.default_rng(4).random(keep.sum())
    kw = model_args(nx, ny, nz, sici, MAXm=M, MAXn=M, seed=9, geometry=geo, rho=rho)
    ora = OracleModel(**kw)
    B = _rhs(ora, nrhs, 3)
    tol = 1e-8
    X, infos = _solve(kw, precision, 8, 12, tol, B)
    A = ora.dense_operator() if ora.N <= 1500 else None
    for k in range(nrhs):
        assert infos[k]["status"] == "converged", infos[k]
        res = np.linalg.norm(B[k] - ora.aproduct_with_alb(X[k])) / np.linalg.norm(B[k])
        assert res <= 1.0001 * tol, (k, res, infos[k])
        assert abs(infos[k]["true_error"] - res) <= 1e-3 * tol, (infos[k]["true_error"], res)
        if A is not None:
            x = np.linalg.solve(A, B[k])
            assert rel(X[k], x) < 1e3 * tol


def test_pgmres_iteration_budget(sici):
    """max_iter bounds the inner operator applications (checked between
    cycles), and the counts in the info are consistent."""
    from oracle.dda_oracle import OracleModel

    kw = model_args(12, 12, 6, sici, MAXm=20, MAXn=20, seed=9)
    B = _rhs(OracleModel(**kw), 1, 1)
    X, infos = _solve(kw, "complex128", 6, 5, 1e-15, B, max_iter=40)
    i = infos[0]
    assert i["status"] == "max_iter", i
    assert i["inner_iterations"] >= i["iterations"] * 6
    # the polynomial's 6 steps, cycles of 5 x 6 checked after every step, the
    # correction's 6, then the budget check
    assert 40 <= i["inner_iterations"] <= 40 + 6 + 6, i


@pytest.mark.parametrize("precision", ["complex128", "mixed"])
@pytest.mark.parametrize("degree,restart,deflate", [(1, 16, 6), (4, 12, 4)])
def test_deflated_restarts_match_oracle(sici, precision, degree, restart, deflate):
    """Deflated restarting (GMRES-DR, harmonic Ritz vectors kept across
    restarts), plain (degree 1) and with the polynomial; short cycles force
    many restarts."""
    from oracle.dda_oracle import OracleModel

    kw = model_args(12, 12, 6, sici, MAXm=20, MAXn=20, seed=4)
    ora = OracleModel(**kw)
    B = _rhs(ora, 2, 8)
    tol = 1e-8
    X, infos = _solve(kw, precision, degree, restart, tol, B, deflate=deflate)
    A = ora.dense_operator()
    for k in range(2):
        assert infos[k]["status"] == "converged", infos[k]
        res = np.linalg.norm(B[k] - ora.aproduct_with_alb(X[k])) / np.linalg.norm(B[k])
        assert res <= 1.0001 * tol, (k, res, infos[k])
        assert rel(X[k], np.linalg.solve(A, B[k])) < 1e3 * tol


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-8), ("mixed", 1e-11), ("complex128", 1e-13)])
@pytest.mark.parametrize("shape,M,nrhs,restart,deflate", [((12, 12, 6), 20, 2, 16, 6), ((16, 16, 8), 50, 1, 24, 10)])
def test_recycled_deflation_space_matches_oracle(sici, precision, tol, shape, M, nrhs, restart, deflate):
    """Solver kind 2: every refinement step after the first starts its inner
    solve from the deflation space the previous one ended with (the new
    residual orthonormalised against it; the cycles then carry the extra
    directions).  Mixed precision takes several refinement steps, so the
    carried space is used; the true residual and the dense solve decide."""
    from oracle.dda_oracle import OracleModel

    nx, ny, nz = shape
    kw = model_args(nx, ny, nz, sici, MAXm=M, MAXn=M, seed=4)
    ora = OracleModel(**kw)
    B = _rhs(ora, nrhs, 8)
    X, infos = _solve(kw, precision, 1, restart, tol, B, deflate=deflate, kind="gmres-dr-recycle")
    A = ora.dense_operator() if ora.N <= 1500 else None
    for k in range(nrhs):
        i = infos[k]
        assert i["status"] == "converged", i
        if precision == "mixed":
            assert i["refinements"] >= 2, i
        res = np.linalg.norm(B[k] - ora.aproduct_with_alb(X[k])) / np.linalg.norm(B[k])
        assert res <= 1.0001 * tol, (k, res, i)
        # the two residual evaluations differ by round-off (~1e-16 relative to ||B||)
        assert abs(i["true_error"] - res) <= max(1e-3 * tol, 1e-15), (i["true_error"], res)
        if A is not None:
            assert rel(X[k], np.linalg.solve(A, B[k])) < 1e4 * tol


def test_recycling_rejects_too_short_cycles(sici):
    from dda_model import DDAModel

    m = DDAModel(**model_args(8, 8, 4, sici, seed=1))
    with pytest.raises(RuntimeError):
        m.setSolver("gmres-dr-recycle", degree=1, restart=10, deflate=6)
    with pytest.raises(RuntimeError):
        m.setSolver("gmres-dr-recycle", degree=1, restart=10, deflate=0)
    m.setSolver("gmres-dr-recycle", degree=1, restart=12, deflate=6)


def test_profile_gram_schmidt(sici):
    """The Gram-Schmidt timing entry point runs both kernels in both precisions
    (odd and even vector lengths: packed and element-wise paths)."""
    from dda_model import DDAModel

    for shape in ((16, 16, 8), (7, 5, 3)):
        m = DDAModel(**model_args(*shape, sici, seed=2), precision="mixed")
        for prec in ("mixed", "complex128"):
            a, b = m.profile_gram_schmidt(prec, nv=9, iters=3)
            assert 0.0 < a < 100.0 and 0.0 < b < 100.0, (shape, prec, a, b)
