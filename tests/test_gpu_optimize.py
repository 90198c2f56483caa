"""The optimisation driver on the GPU: the adjoint-gradient loop against the
reference's finite-difference loop, warm starts, and the output files."""
import numpy as np
import pytest

from cases import model_args

pytestmark = pytest.mark.gpu


def _model(sici, symmetry="None"):
    from dda_model import DDAModel

    # densities kept away from 0, where the reference's one-sided differences
    # of the steep 1/alpha(rho) are inaccurate
    kw = model_args(8, 8, 4, sici, MAXm=1, MAXn=1, symmetry=symmetry, symaxis=(3.5, 3.5), seed=31)
    g = np.asarray(kw["geometry"]).reshape(-1, 3)
    col = np.random.default_rng(32).uniform(0.2, 0.8, (8, 8))
    if symmetry == "4fold":
        col = (col + col[::-1] + col[:, ::-1] + col[::-1, ::-1]) / 4
    kw["inputDielectrics"] = np.repeat(col[g[:, 0], g[:, 1]], 3)
    return DDAModel(**kw)


@pytest.mark.parametrize("symmetry", ["None", "4fold"])
def test_adjoint_loop_tracks_reference_loop(sici, symmetry):
    from dda_model.optimize import TopologyOptimization

    runs = {}
    for grad in ("adjoint", "reference"):
        m = _model(sici, symmetry)
        opt = TopologyOptimization(m, step_size=0.01, penalty_type="parabolic", coeff_type="constant",
                                   coeff_config={"coeff_const": 0.1}, gradient=grad, warm_start=False,
                                   bgs_max_error=1e-10, fd_epsilon=1e-4)
        J0 = opt.objective()
        g = opt.objective_gradient(J0)
        runs[grad] = (g, opt.run(4).objective, m.getParameters())
    ga, gr = runs["adjoint"][0], runs["reference"][0]
    assert ga.shape == gr.shape
    assert np.abs(ga - gr).max() <= 5e-3 * np.abs(ga).max()
    oa, orf = runs["adjoint"][1], runs["reference"][1]
    assert oa[-1] > oa[0]                                   # ascent
    assert np.allclose(oa, orf, rtol=1e-3)
    assert np.abs(runs["adjoint"][2] - runs["reference"][2]).max() < 1e-2


def test_warm_start_and_outputs(sici, tmp_path):
    from dda_model.optimize import TopologyOptimization

    cold = TopologyOptimization(_model(sici), step_size=0.005, warm_start=False, bgs_max_error=1e-8)
    hc = cold.run(5)
    warm = TopologyOptimization(_model(sici), step_size=0.005, warm_start=True, bgs_max_error=1e-8,
                                data_path=str(tmp_path))
    hw = warm.run(5)
    assert np.allclose(hw.objective, hc.objective, rtol=1e-6)
    assert sum(hw.iterations[1:]) < sum(hc.iterations[1:])
    assert np.loadtxt(tmp_path / "Obj.txt").shape == (5,)
    assert np.loadtxt(tmp_path / "Structures" / "Structure4.txt").shape == (3 * 8 * 8 * 4,)


@pytest.mark.parametrize("penalty,cfg,solver", [("parabolic", {}, "reference"),
                                               ("gaussian", {"sigma": 0.3, "mu": 0.5}, "reference"),
                                               ("triangular", {"slope": 1.0}, "jacobi")])
def test_device_loop_follows_host_loop(sici, penalty, cfg, solver):
    """The loop with its state on the GPU (parameters, Adam's averages,
    gradients, penalties) against the host loop: the same objectives and
    parameters, every iteration, for each penalty kind, with the reference's
    BiCGSTAB and with the refinement solver; the symmetric structure exercises
    the parameter map's per-parameter sums."""
    from dda_model.optimize import DeviceTopologyOptimization, TopologyOptimization

    out = {}
    for cls in (TopologyOptimization, DeviceTopologyOptimization):
        m = _model(sici, "4fold")
        if solver == "jacobi":
            m.setPreconditioner("jacobi")
        opt = cls(m, step_size=0.02, penalty_type=penalty, penalty_config=cfg, coeff_type="constant",
                  coeff_config={"coeff_const": 0.2}, warm_start=True, bgs_max_error=1e-10)
        h = opt.run(4)
        out[cls.__name__] = (np.array(h.objective), np.array(h.average_penalty), m.getParameters(),
                             h.iterations)
    (jh, ph, xh, ih), (jd, pd, xd, idv) = out["TopologyOptimization"], out["DeviceTopologyOptimization"]
    assert ih == idv, (ih, idv)                       # the same warm-started solves
    assert np.abs(jd - jh).max() <= 1e-12 * np.abs(jh).max()
    assert np.abs(pd - ph).max() <= 1e-12
    assert np.abs(xd - xh).max() <= 1e-13
    assert jd[-1] != jd[0]
