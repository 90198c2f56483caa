"""The device-driven BiCGSTAB loop: one CUDA graph launch whose while-node
repeats the iterations on the device until every right-hand side is done,
with the iteration budget and a device-side time limit ending it with a
status instead of any host poll.  (Every BiCGSTAB parity test runs through
this loop too: it is the default.)"""
import numpy as np
import pytest

from cases import model_args

pytestmark = pytest.mark.gpu


def test_iteration_budget_ends_the_device_loop(sici):
    from dda_model import DDAModel

    m = DDAModel(**model_args(16, 16, 8, sici, seed=2))
    m.solveElectricField(None, 1, 1e-14)
    info = m.last_solve
    assert info["status"] == "max_iter", info
    assert info["iterations"] <= 1 + 4, info  # stops within one graph body of the budget
    m.solveElectricField(None, 100000, 1e-10)
    assert m.last_solve["status"] == "converged", m.last_solve


@pytest.mark.parametrize("precision", ["complex128", "mixed"])
def test_time_limit_ends_the_device_loop(sici, precision):
    from dda_model import DDAModel

    m = DDAModel(**model_args(48, 48, 12, sici, seed=3, MAXm=50, MAXn=50), precision=precision)
    if precision == "complex128":
        m.setPreconditioner("jacobi")
    m.setTimeLimit(1e-6)
    m.solveElectricField(None, 10**6, 1e-14)
    assert m.last_solve["status"] == "timeout", m.last_solve
    # the model stays usable: without the limit the same solve runs on
    m.setTimeLimit(0.0)
    m.solveElectricField(None, 200, 1e-14)
    assert m.last_solve["status"] in ("max_iter", "converged", "stagnated"), m.last_solve
    assert np.all(np.isfinite(m.getPolarization()))
