"""Serving engine (dda_model.serving over tdda_server_*): every served solve
checked against the oracle's operator (true residual at the requested
tolerance, solution against a dense direct solve), batching and caching
behaviour, and results that do not depend on what else is in flight.

Tolerances: requests are solved to a true relative residual tol; the
solution error is then bounded by cond(A) * tol, checked at 1e3 * tol.
A request solved alone and inside a batch with other requests runs the same
per-right-hand-side arithmetic, checked at 1e-12 relative."""
import numpy as np
import pytest

from cases import model_args, rel

pytestmark = pytest.mark.gpu


def _server(**kw):
    from dda_model.serving import DDAServer

    kw.setdefault("workers", 2)
    kw.setdefault("max_rhs", 8)
    kw.setdefault("hbm_budget_bytes", 8 * 10**9)
    return DDAServer(**kw)


def _request(shape, seed, lam=542.0, theta=0.0, period=0, tol=1e-10, precision="mixed", method="FCD"):
    from dda_model.serving import Request, incidence

    rng = np.random.default_rng(seed)
    nK, pols = incidence(theta)
    return Request(shape=shape, rho=rng.random(int(np.prod(shape))), lam=lam, n_K=nK, polarisations=pols,
                   MAXm=period, MAXn=period, Lm=shape[0] if period else 0.0, Ln=shape[1] if period else 0.0,
                   tol=tol, precision=precision, method=method, tag=seed)


def _check_against_oracle(sici, req, res, sol_tol):
    """True residual with the oracle's operator for each polarisation, the
    internal field, and the solution against a dense direct solve."""
    from oracle.dda_oracle import OracleModel

    nx, ny, nz = req.shape
    for q, e0 in enumerate(req.polarisations):
        kw = model_args(nx, ny, nz, sici, lam=req.lam, d=req.d, material=req.material, MAXm=req.MAXm,
                        MAXn=req.MAXn, Lm=req.Lm or None, Ln=req.Ln or None, method=req.method,
                        n_K=req.n_K, n_E0=e0, rho=req.rho)
        ora = OracleModel(**kw)
        ora.set_densities(req.rho)
        P = res.P[q]
        r = np.linalg.norm(ora.E - ora.aproduct_with_alb(P)) / np.linalg.norm(ora.E)
        assert r <= req.tol * 1.0001, (q, r)
        assert res.info[q]["status"] == "converged"
        assert res.info[q]["true_error"] <= req.tol
        E_int = ora.al * P / ((2.0 + ora.diel) / 3.0)
        assert rel(res.E[q], E_int) < 1e-12
        if ora.N <= 800:
            direct = np.linalg.solve(ora.dense_operator(), ora.E)
            assert rel(P, direct) < sol_tol


@pytest.mark.parametrize("shape,theta,period,method", [
    ((8, 8, 4), 0.0, 0, "FCD"),
    ((8, 6, 4), 25.0, 0, "FCD"),    # oblique: the two polarisations have different 1/alpha
    ((6, 6, 3), 20.0, 1, "FCD"),    # periodic images
    ((7, 5, 3), 10.0, 0, "LDR"),
])
def test_served_solve_matches_oracle(sici, shape, theta, period, method):
    req = _request(shape, seed=1, theta=theta, period=period, method=method)
    with _server(sici=sici) as srv:
        res = srv.solve(req)
    assert res.P.shape == (2, 3 * int(np.prod(shape)))
    _check_against_oracle(sici, req, res, 1e3 * req.tol)


def test_complex128_requests(sici):
    req = _request((8, 8, 4), seed=2, theta=15.0, precision="complex128", tol=1e-11)
    with _server(sici=sici) as srv:
        res = srv.solve(req)
    _check_against_oracle(sici, req, res, 1e3 * req.tol)


def test_same_result_alone_and_in_the_mix(sici):
    """A request gives the same answer alone and when merged into a batch with
    others (same tensor, other designs and angles) while other shapes run
    concurrently on other workers."""
    a = _request((12, 12, 4), seed=3, lam=600.0, theta=12.0)
    with _server(sici=sici, workers=1) as srv:
        alone = srv.solve(a)
        assert alone.batch_requests == 1
    mix = [a]
    mix += [_request((12, 12, 4), seed=10 + i, lam=600.0, theta=3.0 * i) for i in range(3)]   # same key
    mix += [_request((16, 16, 4), seed=20 + i, lam=500.0 + 10 * i) for i in range(3)]          # other shapes
    mix += [_request((8, 8, 8), seed=30 + i, lam=650.0) for i in range(2)]
    with _server(sici=sici, workers=3, max_rhs=8) as srv:
        # hold the workers on other shapes first so that the same-key requests queue up together
        tickets = [srv.submit(r) for r in mix[4:] + mix[:4]]
        results = [srv.wait(t) for t in tickets]
        stats = srv.stats()
    ra = results[len(mix) - 4]
    assert ra.tag == a.tag
    assert stats["completed"] == len(mix)
    assert stats["batches"] < len(mix)          # something was merged
    assert stats["max_concurrent"] >= 2         # batches overlapped on the device
    assert rel(ra.P, alone.P) < 1e-12
    assert rel(ra.E, alone.E) < 1e-12
    for r, res in zip(mix[4:] + mix[:4], results):
        for i in res.info:
            assert i["status"] == "converged" and i["true_error"] <= r.tol


def test_batch_of_different_wavelengths(sici):
    """Same-grid requests with different wavelengths (so different tensors) run
    as one batched solve, each right-hand side with its own tensor; each meets
    its tolerance against the oracle and agrees with its solve alone."""
    reqs = [_request((16, 16, 4), seed=50 + i, lam=480.0 + 60 * i, theta=7.0 * i) for i in range(3)]
    with _server(sici=sici, workers=1) as srv:
        alone = [srv.solve(r) for r in reqs]
    with _server(sici=sici, workers=1) as srv:
        blocker = srv.submit(_request((24, 24, 8), seed=59))
        tickets = [srv.submit(r) for r in reqs]
        srv.wait(blocker)
        mixed = [srv.wait(t) for t in tickets]
    assert [m.batch_requests for m in mixed] == [3, 3, 3]
    assert mixed[0].batch_rhs == 6
    for r, a, m in zip(reqs, alone, mixed):
        assert rel(m.P, a.P) < 1e3 * r.tol
        _check_against_oracle(sici, r, m, 1e3 * r.tol)


def test_tensor_cache_and_eviction(sici):
    from dda_model.serving import DDAServer

    reqs = [_request((16, 16, 4), seed=40, lam=500.0), _request((16, 16, 4), seed=41, lam=520.0),
            _request((16, 16, 4), seed=42, lam=500.0),   # hit
            _request((16, 16, 4), seed=43, lam=540.0),
            _request((16, 16, 4), seed=44, lam=560.0)]
    # room for the workspace and about two tensors of this grid
    probe = DDAServer(hbm_budget_bytes=10**12, workers=1, sici=sici)
    probe.solve(reqs[0])
    ws_and_one = probe.stats()["peak_bytes"]
    probe.close()
    tensor = 17 * 17 * 5 * 6 * 24  # folded 32x32x8 tensor, complex128 + complex64
    with DDAServer(hbm_budget_bytes=ws_and_one + tensor + tensor // 2, workers=1, sici=sici) as srv:
        out = [srv.solve(r) for r in reqs]
        st = srv.stats()
    assert [o.cache_hit for o in out] == [False, False, True, False, False]
    assert st["evictions"] >= 2
    assert st["peak_bytes"] <= ws_and_one + tensor + tensor // 2
    for r, o in zip(reqs, out):
        for i in o.info:
            assert i["status"] == "converged" and i["true_error"] <= r.tol


def test_oversized_request_is_refused(sici):
    from dda_model import TddaError

    with _server(sici=sici, hbm_budget_bytes=10**6) as srv:
        with pytest.raises(TddaError):
            srv.submit(_request((16, 16, 4), seed=5))


def test_graph_replay_matches_direct_launches(sici):
    req = _request((16, 16, 8), seed=6, theta=5.0)
    with _server(sici=sici, use_graphs=False) as srv:
        plain = srv.solve(req)
    with _server(sici=sici, use_graphs=True, graph_steps=4) as srv:
        graph = srv.solve(req)
    assert plain.info[0]["iterations"] == graph.info[0]["iterations"]
    assert rel(graph.P, plain.P) < 1e-14


def test_stream_of_mixed_requests(sici):
    """A short Poisson stream over the four serving grids: every request meets
    its tolerance, latency percentiles are reported."""
    from dda_model.serving import run_stream, synthetic_stream

    reqs = synthetic_stream(n=24, rate=400.0, seed=8)
    with _server(sici=sici, workers=4, hbm_budget_bytes=40 * 10**9) as srv:
        rep = run_stream(srv, reqs)
        st = srv.stats()
    s = rep.summary()
    assert s["requests"] == 24 and s["converged_rhs"] == 48
    assert s["max_true_error"] <= 1e-8
    assert s["p99_ms"] >= s["p50_ms"] > 0
    assert st["completed"] == 24 and st["failed"] == 0


def test_invalid_requests_and_tickets(sici):
    """Bad requests fail at submit with a message; unknown tickets and
    timeouts are reported, not waited on forever."""
    import ctypes

    from dda_model import TddaError, _lib
    from dda_model.serving import Request

    with _server(sici=sici, workers=1) as srv:
        good = _request((8, 8, 4), seed=60)
        bad = [
            Request(shape=(8, 8, 4), rho=np.full(256, 1.5)),                        # density outside [0, 1]
            Request(shape=(8, 8, 4), rho=np.zeros(256), polarisations=((1, 0, 0),) * 5),  # > 4 polarisations
            Request(shape=(8, 8, 4), rho=np.zeros(256), tol=0.0),
            Request(shape=(8, 8, 4), rho=np.zeros(256), lam=-1.0),
        ]
        for r in bad:
            with pytest.raises((TddaError, ValueError, IndexError)):
                srv.submit(r)
        with pytest.raises(ValueError):
            srv.submit(Request(shape=(8, 8, 4), rho=np.zeros(10)))             # wrong size
        res = _lib.RequestResult()
        assert srv._lib.tdda_server_wait(srv._h, 987654, 0.0, ctypes.byref(res)) == 1  # unknown ticket
        t = srv.submit(good)
        out = srv.wait(t)
        assert out.info[0]["status"] == "converged"
        assert srv._lib.tdda_server_wait(srv._h, t, 0.0, ctypes.byref(res)) == 1       # waited for once
        st = srv.stats()
        assert st["submitted"] == 1 and st["completed"] == 1 and st["failed"] == 0


def test_shutdown_finishes_queued_work(sici):
    """Closing the server with requests still queued finishes them first (their
    output buffers are filled) and then returns."""
    import ctypes

    from dda_model import _lib
    from dda_model.serving import DDAServer

    srv = DDAServer(hbm_budget_bytes=8 * 10**9, workers=1, sici=sici)
    reqs = [_request((12, 12, 4), seed=70 + i, lam=500.0 + 20 * i) for i in range(4)]
    tickets = [srv.submit(r) for r in reqs]
    # a zero timeout on the last request, which cannot have finished yet, reports TIMEOUT
    res = _lib.RequestResult()
    assert srv._lib.tdda_server_wait(srv._h, tickets[-1], 0.0, ctypes.byref(res)) in (0, 6)
    outputs = [srv._pending[t][1] for t in tickets]
    srv.close()
    assert all(np.abs(P).max() > 0 for P in outputs)


def test_reserved_workspaces(sici):
    """Reserving a grid allocates every worker's workspace up front (counted
    in the budget); requests of that grid then run without allocating."""
    from dda_model import TddaError

    with _server(sici=sici, workers=2) as srv:
        before = srv.stats()["bytes_in_use"]
        srv.reserve((16, 16, 4))
        after = srv.stats()["bytes_in_use"]
        assert after > before
        res = srv.solve(_request((16, 16, 4), seed=80))
        assert res.info[0]["status"] == "converged"
        assert srv.stats()["bytes_in_use"] >= after   # plus the request's tensor
        srv.reserve((16, 16, 4))                      # already there: no change
    with _server(sici=sici, workers=2, hbm_budget_bytes=10**7) as srv:
        with pytest.raises(TddaError):
            srv.reserve((64, 64, 16))
