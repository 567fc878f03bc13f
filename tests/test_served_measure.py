"""The served leg's comparison (CPU only): the highest sustainable arrival
rate at a p99 bound, interpolated from a sweep, and the engine-to-plain
ratio at the plain path's own p99 bounds."""
import pytest

import bench


def test_sustainable_rate_interpolates_first_crossing():
    pts = [(100, 10.0), (200, 20.0), (300, 40.0)]
    assert bench.sustainable_rate(pts, 30.0) == pytest.approx(250.0)
    assert bench.sustainable_rate(pts, 40.0) == 300           # no crossing: the top swept rate
    assert bench.sustainable_rate(pts, 5.0) is None            # the lowest rate already misses the bound
    # a later dip below the bound after the first crossing does not count
    assert bench.sustainable_rate([(100, 10.0), (200, 60.0), (300, 20.0)], 35.0) == pytest.approx(150.0)
    assert bench.sustainable_rate(list(reversed(pts)), 30.0) == pytest.approx(250.0)  # order does not matter


def test_equal_p99_rates_uses_plain_bounds():
    cap = 500.0
    plain = [{"rate": m * cap, "p99_ms": p} for m, p in [(0.5, 30), (0.6, 33), (0.7, 38), (0.8, 45), (0.85, 48),
                                                          (0.9, 54), (0.95, 62)]]
    eng = [{"rate": m * cap, "p99_ms": p} for m, p in [(0.5, 25), (0.7, 35), (0.9, 44), (1.0, 51), (1.2, 66)]]
    out = bench.equal_p99_rates(plain, eng, cap)
    assert set(out) == {"plain_p99_at_0.8x_capacity", "plain_p99_at_0.9x_capacity", "plain_p99_at_0.95x_capacity"}
    b = out["plain_p99_at_0.8x_capacity"]
    assert b["p99_bound_ms"] == 45 and b["plain_rate_per_s"] == pytest.approx(400.0)
    assert b["engine_rate_per_s"] == pytest.approx(450 + 1 / 7 * 50)  # between (0.9, 44) and (1.0, 51)
    assert b["ratio"] == pytest.approx(b["engine_rate_per_s"] / 400.0)
