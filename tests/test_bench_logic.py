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


def test_cone_roofline_points_are_interior():
    """The cone-kernel workload's s and z are strictly inside their cones
    (and the power cones' z inside the dual cone for the same alphas)."""
    rng = np.random.default_rng(3)
    v, _ = bench.cone_points(1, 1000, 1, rng)
    assert v.min() > 0
    v, _ = bench.cone_points(2, 10, 500, rng)
    V = v.reshape(-1, 10)
    assert np.all(V[:, 0] > np.linalg.norm(V[:, 1:], axis=1))
    v, _ = bench.cone_points(3, 3, 500, rng)
    x, y, z = v.reshape(-1, 3).T
    assert np.all(y > 0) and np.all(y * np.exp(x / y) < z)            # primal exp cone
    assert np.all(x < 0) and np.all(-x * np.exp(y / x) < np.e * z)     # dual exp cone
    s, a = bench.cone_points(4, 3, 500, rng)
    zz, _ = bench.cone_points(4, 3, 500, rng, a)
    S, Z = s.reshape(-1, 3), zz.reshape(-1, 3)
    assert np.all(S[:, 0] ** a * S[:, 1] ** (1 - a) > np.abs(S[:, 2]))
    assert np.all((Z[:, 0] / a) ** a * (Z[:, 1] / (1 - a)) ** (1 - a) > np.abs(Z[:, 2]))
    v, _ = bench.cone_points(5, 10, 50, rng)
    n, t = 10, 55
    ii, jj = np.triu_indices(n)
    order = np.lexsort((ii, jj))  # svec: column by column, upper triangle
    for x in v.reshape(-1, t):
        M = np.zeros((n, n))
        vals = x / np.where(ii[order] == jj[order], 1.0, np.sqrt(2.0))
        M[ii[order], jj[order]] = vals
        M = M + np.triu(M, 1).T
        assert np.linalg.eigvalsh(M).min() > 0
