"""The allocation-free operator entry point (tdda_matvec_device_noalloc).

It serves callers that cannot have device memory allocated while a call runs
(fixed device-memory budgets, latency-bound host threads): it works only in
the caller's buffers and a fixed scratch array inside the library.  Here it
must give the same result as the ordinary device matvec and as the oracle,
call after call (the scratch keeps the previous call's contents), leave the
device's free memory unchanged once warmed up, and reject grids too large for
the scratch.  The file name sorts last so that a run stopped at its first
failure (pytest -x) has already run every other test when a failure of this
optional entry point stops it; the tests do not depend on running last.
"""
import numpy as np
import pytest

from cases import model_args, rel

pytestmark = pytest.mark.gpu


def _vec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


@pytest.mark.parametrize("shape,periodic,subset", [((16, 16, 8), 0, False), ((12, 10, 6), 2, False),
                                                   ((10, 9, 4), 1, True)])
def test_noalloc_matches_device_matvec_twice(sici, shape, periodic, subset):
    import torch

    from dda_model import DDAModel
    from oracle.dda_oracle import generate_geometry

    nx, ny, nz = shape
    geo = None
    rho = None
    if subset:  # dipoles on part of the box: cells without a dipole must stay zero
        g = generate_geometry(nx, ny, nz).reshape(-1, 3)
        keep = (g[:, 0] + g[:, 1]) % 3 != 0
        geo = g[keep].ravel()
        rho = np.linspace(0.1, 0.9, keep.sum())
    m = DDAModel(**model_args(nx, ny, nz, sici, MAXm=periodic, MAXn=periodic, seed=3, geometry=geo, rho=rho))
    n3 = 3 * m.N
    s = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((1, 2)):
        x = torch.from_numpy(_vec(n3, seed)).cuda()
        y_ref = torch.zeros_like(x)
        y = torch.zeros_like(x)
        m.matvec_device(x.data_ptr(), y_ref.data_ptr(), 1, True, s)
        m.matvec_device_noalloc(x.data_ptr(), y.data_ptr(), True, s)
        torch.cuda.synchronize()
        assert rel(y.cpu().numpy(), y_ref.cpu().numpy()) < 1e-13, f"call {call}"
        # without the polarisability term too
        m.matvec_device(x.data_ptr(), y_ref.data_ptr(), 1, False, s)
        m.matvec_device_noalloc(x.data_ptr(), y.data_ptr(), False, s)
        torch.cuda.synchronize()
        assert rel(y.cpu().numpy(), y_ref.cpu().numpy()) < 1e-13, f"call {call}"


def test_noalloc_rejects_grids_beyond_its_scratch(sici):
    import torch

    from dda_model import DDAModel
    from dda_model._lib import TddaError

    m = DDAModel(**model_args(64, 64, 32, sici, seed=1))  # needs 36 MiB > 32 MiB
    x = torch.zeros(3 * m.N, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    with pytest.raises(TddaError, match="MiB of scratch"):
        m.matvec_device_noalloc(x.data_ptr(), y.data_ptr(), True, torch.cuda.current_stream().cuda_stream)


def test_noalloc_matches_oracle_and_allocates_nothing(sici):
    """Two calls in a row against the oracle's A.x (+ 1/alpha), and no change
    of the device's free memory across calls after one warm-up call (which may
    load the grid's kernels)."""
    import torch

    from dda_model import DDAModel
    from oracle.dda_oracle import OracleModel

    kw = model_args(12, 10, 6, sici, MAXm=2, MAXn=2, seed=5)
    m = DDAModel(**kw)
    ora = OracleModel(**kw)
    n3 = 3 * m.N
    s = torch.cuda.current_stream().cuda_stream
    xs = [torch.from_numpy(_vec(n3, seed)).cuda() for seed in (7, 8)]
    ys = [torch.zeros_like(xs[0]) for _ in range(2)]
    m.matvec_device_noalloc(xs[0].data_ptr(), ys[0].data_ptr(), True, s)  # warm-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        for x, y in zip(xs, ys):
            m.matvec_device_noalloc(x.data_ptr(), y.data_ptr(), True, s)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for x, y in zip(xs, ys):
        xh = x.cpu().numpy()
        assert rel(y.cpu().numpy(), ora.aproduct_with_alb(xh)) < 1e-12
