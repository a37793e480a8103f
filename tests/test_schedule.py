"""The runtime's step schedule without a GPU: ``plan_steps`` (integer-microsecond
arrays) gives, step for step, the cursor walk of the oracle's restatement of
``main._run`` (main.py:1383-1389, 1610) — the same cursor instants, float64 cursor
offsets, step lengths (the last one cut to end on the terminus), hourly windows and
RK2 weights alpha (main.py:916-919) — on the golden runs' schedules and on seeded
random ones (odd step lengths, unaligned instants, spans shorter than a step, empty
walks); and ``schedule_array`` / ``window_ranges`` follow from it."""

from __future__ import annotations

from datetime import UTC, datetime, timedelta

import numpy as np
import pytest

from fixtures import load_run
from oracle import runtime as ort


def oracle_walk(batch_start, cursor_start, terminus, dt_s):
    """The schedule part of oracle.runtime.run_batch's loop."""
    out = []
    t = cursor_start
    b = batch_start.timestamp()
    while t > terminus:
        delta = min(float(dt_s), (t - terminus).total_seconds())
        hk = ort.hour_floor(t)
        alpha = ort.advection_alpha(hk, hk + timedelta(hours=1), t, delta)
        out.append((t, t.timestamp() - b, delta, hk, alpha))
        t = t - timedelta(seconds=delta)
    return out


def _check(batch_start, cursor_start, terminus, dt_s):
    from glide_b200.runtime import plan_steps, schedule_array, window_ranges

    want = oracle_walk(batch_start, cursor_start, terminus, dt_s)
    got = plan_steps(batch_start, cursor_start, terminus, dt_s)
    assert len(got) == len(want)
    for k, (s, w) in enumerate(zip(got, want)):
        assert s.cursor == w[0], k
        assert s.cursor_off == w[1], k
        assert s.delta == w[2], k
        assert s.hour == w[3], k
        assert s.alpha == w[4], k
    rec = schedule_array(got)
    np.testing.assert_array_equal(rec["c"], np.array([w[1] for w in want], dtype=np.float32))
    np.testing.assert_array_equal(rec["d"], np.array([w[2] for w in want], dtype=np.float32))
    np.testing.assert_array_equal(rec["a"], np.array([w[4] for w in want], dtype=np.float32))
    np.testing.assert_array_equal(rec["i"], np.arange(len(want)))
    ranges = window_ranges(got)
    assert [want[e - 1][3] == want[k][3] for k, e in ranges] == [True] * len(ranges)
    assert sum(e - k for k, e in ranges) == len(want)
    assert all(want[e][3] != want[e - 1][3] for _, e in ranges[:-1])
    return len(want)


@pytest.mark.parametrize("name", ["run_small", "run_c0"])
def test_golden_run_schedules(name):
    run = load_run(name)
    n = _check(run.dt_("batch_start"), run.dt_("cursor_start"), run.dt_("cursor_terminus"), float(run.z["dt_s"]))
    if "n_steps" in run.z:
        assert n == int(run.z["n_steps"])
    assert n == run.z["out_active"].size


def test_random_schedules():
    rng = np.random.default_rng(20261203)
    base = datetime(2024, 1, 15, tzinfo=UTC)
    for _ in range(40):
        dt_s = float(rng.choice([30.0, 60.0, 7.5, 30.0000001, 0.1 * 3, 900.0]))
        start = base + timedelta(microseconds=int(rng.integers(0, 86_400_000_000)))
        span = timedelta(microseconds=int(rng.integers(1, 3 * 3_600_000_000 if dt_s > 1 else 30_000_000)))
        batch_start = start - timedelta(hours=int(rng.integers(0, 48)))
        _check(batch_start, start, start - span, dt_s)


def test_edge_schedules():
    t = datetime(2024, 1, 15, 12, 0, 0, tzinfo=UTC)
    assert _check(t, t, t, 30.0) == 0  # empty walk
    assert _check(t, t, t + timedelta(seconds=5), 30.0) == 0  # terminus after the start
    assert _check(t, t, t - timedelta(seconds=10), 30.0) == 1  # one short step
    assert _check(t, t, t - timedelta(hours=1), 30.0) == 120  # hour-aligned: one window
    # 7200 s + 4 us: 240 full steps and a 4 us one, across three hourly windows
    assert _check(t, t + timedelta(microseconds=1), t - timedelta(hours=2, microseconds=3), 30.0) == 241
