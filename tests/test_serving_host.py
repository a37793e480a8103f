"""The serving workload's request stream without a GPU: ``poisson_requests`` is
seeded and reproducible, its arrivals are a Poisson process of the asked rate, and
sites, release times, particle counts and durations stay in the ranges the serving
workload names (56 sites, release times in whole minutes within the window, N
log-uniform in [1e3, 5e4], 6-120 h)."""

from __future__ import annotations

from datetime import UTC, datetime, timedelta

import numpy as np


def test_poisson_request_stream():
    from glide_b200.serving import poisson_requests

    rng = np.random.default_rng(3)
    sites = np.stack([rng.uniform(-50.0, 30.0, 56), rng.uniform(20.0, 70.0, 56)], axis=1)
    t0 = datetime(2024, 1, 3, tzinfo=UTC)
    reqs = poisson_requests(2000, 5.0, sites, t0, 48.0, seed=20261207)
    again = poisson_requests(2000, 5.0, sites, t0, 48.0, seed=20261207)
    assert reqs == again
    assert poisson_requests(5, 5.0, sites, t0, 48.0, seed=1) != poisson_requests(5, 5.0, sites, t0, 48.0, seed=2)
    arr = np.array([r.arrival_s for r in reqs])
    gaps = np.diff(np.concatenate([[0.0], arr]))
    assert np.all(gaps > 0)
    # mean gap 0.2 s (rate 5/s) within 5 standard errors; exponential: std == mean
    assert abs(gaps.mean() - 0.2) < 5 * 0.2 / np.sqrt(gaps.size)
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.1
    site_set = {(float(s[0]), float(s[1])) for s in sites}
    assert all((r.lon, r.lat) in site_set for r in reqs)
    rel = np.array([(r.release_time - t0) / timedelta(minutes=1) for r in reqs])
    assert np.all(rel == np.floor(rel)) and rel.min() >= 0 and rel.max() < 48 * 60
    n = np.array([r.n_particles for r in reqs])
    assert n.min() >= 1000 and n.max() <= 50000
    # log-uniform: the median near the geometric mean of the range
    assert abs(np.log(np.median(n)) - 0.5 * (np.log(1000) + np.log(50000))) < 0.2
    dur = np.array([r.duration_h for r in reqs])
    assert dur.min() >= 6.0 and dur.max() <= 120.0
    assert all(10.0 <= r.height_m <= 300.0 for r in reqs)
    assert [r.request_id for r in reqs] == list(range(2000))
