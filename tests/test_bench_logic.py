"""Host-side arithmetic of bench.py (no GPU): the plain path's latency under
the served run's arrival stream, and the cone operations' byte counts."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_plain_under_load_matches_a_hand_computed_fifo_queue():
    # same arrivals as the served run: replay the generator by hand
    rng = np.random.default_rng(5)
    n = int(rng.poisson(50 * 2.0))
    arrive = np.sort(rng.uniform(0.0, 2.0, n))
    svc = [0.01, 0.03]
    t, resp = 0.0, []
    for i in range(n):
        t = max(t, arrive[i]) + svc[i % 2]
        resp.append(t - arrive[i])
    r = bench.plain_under_load(svc, 50, 2.0, 5)
    assert r["requests"] == n
    assert abs(r["p50_ms"] - 1000 * np.percentile(resp, 50)) < 1e-9
    assert abs(r["p99_ms"] - 1000 * np.percentile(resp, 99)) < 1e-9


def test_plain_under_load_saturates_when_arrivals_outpace_service():
    r = bench.plain_under_load([0.0075], 2000, 1.0, 1)
    # ~2000 requests at 133/s: the last waits ~14 s
    assert r["p99_ms"] > 10000 and r["value"] < 140


def test_cone_op_bytes_per_element_and_cone():
    assert bench.cone_op_bytes("update_scaling", 1, 1000, 1) == 32 * 1000
    # sparse SOC(10): 32 B/row + 8 B/cone, + 16 B/row (u, v) + 8 B/cone (d)
    assert bench.cone_op_bytes("update_scaling", 2, 10, 3) == 3 * (48 * 10 + 16)
    assert bench.cone_op_bytes("mul_Hs", 3, 3, 5) == 5 * 120
    assert bench.cone_op_bytes("step_length", 4, 3, 2) == 2 * 104
    # PSD(10): svec 55 entries, R and R^-1 100 entries each, lambda 10
    assert bench.cone_op_bytes("update_scaling", 5, 10, 1) == 16 * 55 + 16 * 100 + 8 * 10
