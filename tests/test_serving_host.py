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
