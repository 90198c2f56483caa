"""Host-side logic of the serving loop (no GPU): the synthetic request stream
and the incidence geometry."""
import math

import numpy as np


def test_incidence_polarisations_are_transverse():
    from dda_model.serving import incidence

    for theta in (0.0, 12.5, 30.0):
        nK, (p, s) = incidence(theta)
        assert abs(np.linalg.norm(nK) - 1) < 1e-15
        assert abs(np.dot(nK, p)) < 1e-15 and abs(np.dot(nK, s)) < 1e-15
        assert abs(np.dot(p, s)) < 1e-15
        assert abs(math.degrees(math.acos(nK[2])) - theta) < 1e-9


def test_synthetic_stream_shapes_and_arrivals():
    from dda_model.serving import SERVE_SHAPES, synthetic_stream

    reqs = synthetic_stream(n=512, rate=200.0, seed=7)
    assert len(reqs) == 512
    t = np.array([r.arrival_s for r in reqs])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 200.0) < 0.15 / 200.0          # Poisson at 200 req/s
    counts = {s: 0 for s in SERVE_SHAPES}
    for r in reqs:
        counts[r.shape] += 1
        assert r.rho.size == np.prod(r.shape) and r.rho.min() >= 0 and r.rho.max() <= 1
        assert 450.0 <= r.lam <= 700.0
        assert len(r.polarisations) == 2
        assert math.degrees(math.acos(r.n_K[2])) <= 30.0 + 1e-9
    assert min(counts.values()) > 512 / 4 * 0.7
    # seeded: the same stream twice
    again = synthetic_stream(n=512, rate=200.0, seed=7)
    assert all(a.lam == b.lam and np.array_equal(a.rho, b.rho) for a, b in zip(reqs, again))


def test_per_grid_service_summary():
    """Per-grid record of a stream: each batch counted once however many
    requests it merged, service seconds summed per batch."""
    from dda_model.serving import Result, StreamReport, synthetic_stream

    reqs = synthetic_stream(n=6, rate=100.0, seed=3)
    shapes = [r.shape for r in reqs]
    res = []
    for i, sh in enumerate(shapes):
        merged = 2 if i < 2 else 1          # the first two requests share one 4-RHS batch
        res.append(Result(P=None, E=None, info=[{"inner_iterations": 10 + i, "status": "converged",
                                                 "true_error": 1e-9}] * 2,
                          batch_rhs=2 * merged, batch_requests=merged, cache_hit=False, worker=0, queue_ms=0.0,
                          build_ms=0.0, solve_ms=50.0, total_ms=60.0))
    rep = StreamReport(results=res, requests=reqs, wall_s=1.0)
    per = rep.per_shape()
    assert sum(v["requests"] for v in per.values()) == 6
    assert abs(sum(v["batches"] for v in per.values()) - 5.0) < 1e-12   # 6 requests in 5 batches
    assert abs(sum(v["solve_s_total"] for v in per.values()) - 0.25) < 1e-12
    for key, v in per.items():
        assert key.count("x") == 2
        assert v["median_batch_solve_ms"] == 50.0
