"""Host logic of the serving loop (no GPU): arrival processes, the admission
budget and the latency percentiles."""

from __future__ import annotations

import numpy as np

from cujpegxl_b200.serve import DEFAULT_STREAMS, Budget, frame_seed, latency_stats, percentile, poisson_arrivals


def test_poisson_arrivals_rate_order_and_seed():
    rng = np.random.Generator(np.random.PCG64(0))
    t = poisson_arrivals(60.0, 100.0, rng)
    assert np.all(np.diff(t) > 0) and t[0] >= 0 and t[-1] < 100.0
    assert abs(len(t) - 6000) < 4 * np.sqrt(6000)
    gaps = np.diff(t)
    assert abs(gaps.mean() - 1 / 60.0) < 0.05 / 60.0
    again = poisson_arrivals(60.0, 100.0, np.random.Generator(np.random.PCG64(0)))
    np.testing.assert_array_equal(t, again)
    assert len(poisson_arrivals(0.0, 10.0, rng)) == 0


def test_budget_admits_until_full_and_releases():
    b = Budget(100)
    assert b.reserve(60)
    assert not b.reserve(41)
    assert b.reserve(40)
    b.release(60)
    assert b.used == 40 and b.reserve(60)


def test_percentiles():
    assert percentile([], 50) is None
    v = list(range(101))
    assert percentile(v, 50) == 50 and percentile(v, 99) == 99 and percentile(v, 100) == 100
    # Index llround(p * (n - 1)) as in the reference's benchmark: halves round up.
    assert percentile([1.0, 2.0], 50) == 2.0
    assert percentile(list(range(4)), 50) == 2


def test_latency_stats_match_the_reference_benchmark_set():
    s = latency_stats([3.0, 1.0, 2.0, 4.0])
    assert s["n"] == 4 and s["mean"] == 2.5 and s["min"] == 1.0 and s["max"] == 4.0
    assert abs(s["stddev"] - (5.0 / 3.0) ** 0.5) < 1e-12
    assert s["p50"] == 3.0 and s["p99"] == 4.0
    assert latency_stats([]) == {"n": 0}


def test_frame_seeds_are_distinct_across_streams_and_frames():
    seeds = {frame_seed(i, k) for i in range(8) for k in range(4)}
    assert len(seeds) == 32


def test_default_workload_matches_the_serving_configuration():
    kinds = [(s.width, s.height, s.fps) for s in DEFAULT_STREAMS]
    assert kinds.count((3840, 2160, 30.0)) == 2
    assert kinds.count((1920, 1080, 60.0)) == 4
    assert kinds.count((1280, 720, 60.0)) == 2
