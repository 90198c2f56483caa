"""The design-density kernels (cone filter + tanh projection and their
adjoints, tdda_design_forward_device / tdda_design_backward_device) against
the elementwise numpy/torch evaluation in dda_model.filters, and the device
path of the differentiable objective against the host path.

Tolerances: the forward pass evaluates the same sums in the same order with
every product and sum rounded separately, so the filtered field is checked
bit-equal; the projection uses the device tanh (a few ulp from the host's),
checked at 1e-14.  The backward pass is checked against torch autograd of the
elementwise filter at 1e-12 relative (different summation order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,radius", [((12, 10, 6), 2.0), ((7, 9, 3), 1.5), ((16, 16, 8), 3.0),
                                          ((5, 4, 1), 2.0)])
def test_design_forward_backward(shape, radius):
    import torch

    from dda_model import filters
    from dda_model.autograd import design_densities

    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 100 + ny)
    raw = rng.random(shape)
    beta, eta = 8.0, 0.5
    x = torch.tensor(raw, dtype=torch.float64, device="cuda", requires_grad=True)
    rho = design_densities(x, radius, beta, eta)
    f_np = filters.cone_filter(raw, radius)
    rho_np = filters.dipole_order(np.clip(filters.tanh_projection(f_np, beta, eta), 0.0, 1.0))
    assert np.max(np.abs(rho.detach().cpu().numpy() - rho_np)) <= 1e-14
    w = rng.standard_normal(nx * ny * nz)
    (rho * torch.tensor(w, device="cuda")).sum().backward()
    xt = torch.tensor(raw, dtype=torch.float64, requires_grad=True)
    pt = filters.tanh_projection(filters.cone_filter(xt, radius), beta, eta).clamp(0.0, 1.0)
    (pt.permute(2, 1, 0).reshape(-1) * torch.tensor(w)).sum().backward()
    g_dev = x.grad.cpu().numpy()
    g_ref = xt.grad.numpy()
    assert np.linalg.norm(g_dev - g_ref) <= 1e-12 * np.linalg.norm(g_ref)


def test_filtered_field_is_bit_equal():
    import torch

    from dda_model import _lib, filters

    nx, ny, nz = 9, 8, 5
    raw = np.random.default_rng(1).random((nx, ny, nz))
    x = torch.tensor(raw, device="cuda")
    f = torch.empty_like(x)
    r = torch.empty(nx * ny * nz, dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().tdda_design_forward_device(nx, ny, nz, 2.0, 8.0, 0.5, x.data_ptr(), f.data_ptr(),
                                                      r.data_ptr(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert np.array_equal(f.cpu().numpy(), filters.cone_filter(raw, 2.0))


def test_design_rejects_bad_arguments():
    import torch

    from dda_model import _lib
    from dda_model._lib import TddaError

    x = torch.zeros((4, 4, 4), dtype=torch.float64, device="cuda")
    f = torch.empty_like(x)
    r = torch.empty(64, dtype=torch.float64, device="cuda")
    with pytest.raises(TddaError, match="radius"):
        _lib.check(_lib.load().tdda_design_forward_device(4, 4, 4, 7.0, 8.0, 0.5, x.data_ptr(), f.data_ptr(),
                                                          r.data_ptr(), None))


def test_device_objective_path_matches_host_path(sici):
    """The autograd objective with CUDA densities (device pointers in and out)
    gives the same value and gradient as with CPU densities (host arrays)."""
    import torch

    from cases import model_args
    from dda_model import DDAModel
    from dda_model.autograd import dda_objective

    nx, ny, nz = 10, 8, 4
    m = DDAModel(**model_args(nx, ny, nz, sici, MAXm=2, MAXn=2, seed=3))
    m.setObservationPoints(np.array([[x, y, nz + 1] for x in range(3, 6) for y in range(2, 5)]))
    rho0 = np.random.default_rng(2).random(nx * ny * nz)
    out = {}
    for dev in ("cpu", "cuda"):
        for kind in ("patch", "integrated"):
            r = torch.tensor(rho0, device=dev, requires_grad=True)
            J = dda_objective(r, m, kind=kind, tol=1e-12)
            J.backward()
            out[(dev, kind)] = (float(J), r.grad.cpu().numpy())
    for kind in ("patch", "integrated"):
        Jc, gc = out[("cpu", kind)]
        Jd, gd = out[("cuda", kind)]
        assert abs(Jc - Jd) <= 1e-12 * abs(Jc)
        assert np.linalg.norm(gc - gd) <= 1e-9 * np.linalg.norm(gc)
    # densities set on the device are what getDielectrics reports
    r = torch.tensor(rho0, device="cuda")
    m.setDensitiesDevice(r.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert np.array_equal(m.getDielectrics()[0::3], rho0)
    with pytest.raises(Exception, match="outside"):
        bad = r.clone()
        bad[3] = 1.5
        m.setDensitiesDevice(bad.data_ptr(), torch.cuda.current_stream().cuda_stream)
