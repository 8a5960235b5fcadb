"""Host-side logic of bench.py and of the serving lanes (no GPU): the lanes'
slot protocol, budget admission and concurrency on fake solvers, and the
cone operations' byte counts."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class _Status:
    name = "SOLVED"


class _Sol:
    status = _Status()

    def __init__(self, it):
        self.iterations = it


class FakeSlots:
    """The serve_* protocol of BatchSolver on the host: an admitted slot
    joins the next step and finishes after `steps[slot]` steps."""

    def __init__(self, steps, nbytes=1000):
        self.steps, self.left, self.nbytes = steps, {}, nbytes
        self.admitted = []

    def device_bytes(self):
        return self.nbytes

    def serve_admit(self, slots, q=None, b=None, stream=0):
        for k in slots:
            assert k not in self.left, "slot admitted while running"
            self.left[k] = self.steps[k]
            self.admitted.append(k)

    def serve_step(self, stream=0):
        fin = []
        for k in list(self.left):
            self.left[k] -= 1
            if self.left[k] == 0:
                fin.append(k)
                del self.left[k]
        return sorted(fin), len(self.left)

    def serve_collect(self, slots, stream=0):
        return [_Sol(self.steps[k]) for k in slots]


def test_slot_lane_serves_every_request_in_slot_order():
    from cuclarabel_b200 import serving
    budget = serving.Budget(10_000)
    fake = FakeSlots({0: 3, 1: 5, 2: 2})
    lane = serving.SlotLane("fake", fake, 0, budget)
    assert budget.held == 1000
    arrive = np.zeros(7)
    slot = np.array([0, 1, 0, 2, 0, 1, 2])
    left = lane.run(0.0 + __import__("time").perf_counter(), arrive, slot, [None] * 7,
                    [None] * 7, 30.0)
    assert left == 0 and len(lane.stats.lat) == 7
    # a slot's requests run one after another, in arrival order
    assert [k for k in fake.admitted if k == 0] == [0, 0, 0]
    assert lane.stats.status["SOLVED"] == 7
    lane.close()
    assert budget.held == 0


def test_cohort_lane_waits_for_the_budget_and_frees_it():
    from cuclarabel_b200 import serving
    import scipy.sparse as sp
    budget = serving.Budget(5000)
    budget.hold(4000)  # a resident lane
    made = []

    def make(pbs):
        made.append(len(pbs))
        return FakeSlots({k: 2 for k in range(len(pbs))}, nbytes=800)

    lane = serving.CohortLane("fake", 0, budget, bytes_per_nnz=1.0, make_solver=make)
    pb = (sp.csc_matrix((3, 3)), np.zeros(3), sp.csc_matrix(np.eye(3)), np.zeros(3), [])
    import threading
    import time
    t0 = time.perf_counter()
    # 9 nnz per problem: 4 problems need 36 + 4000 <= 5000; then true 800 B
    th = threading.Thread(target=lambda: lane.run(t0, np.zeros(4), [pb] * 4, 30.0))
    th.start()
    th.join(10)
    assert not th.is_alive()
    assert made == [4] and lane.cohorts == 1 and len(lane.stats.lat) == 4
    assert budget.held == 4000 and budget.peak == 4800
    # a cohort larger than the free budget waits until the horizon
    budget.hold(950)
    lane2 = serving.CohortLane("fake", 0, budget, bytes_per_nnz=100.0, make_solver=make)
    left = lane2.run(time.perf_counter(), np.zeros(2), [pb] * 2, 0.05)
    assert left == 2 and lane2.waited_for_budget > 0 and lane2.cohorts == 0


def test_run_lanes_runs_lanes_concurrently():
    from cuclarabel_b200 import serving

    class Sleeper:
        def run(self, t0, d, horizon):
            import time
            time.sleep(d)
            return 0

    wall, left = serving.run_lanes([(Sleeper(), (0.2,)), (Sleeper(), (0.2,))], 5.0)
    assert left == [0, 0] and wall < 0.35


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


def test_slot_lane_warm_serves_one_request_outside_the_stats():
    from cuclarabel_b200 import serving
    fake = FakeSlots({0: 2, 1: 3})
    lane = serving.SlotLane("fake", fake, 0, serving.Budget(10_000))
    lane.warm(1)
    assert fake.admitted == [1] and not fake.left and lane.stats.lat == []


def test_mixed_precision_error_summary():
    """obj_errors compares only instances converged by the run (SOLVED or
    ALMOST_SOLVED) and SOLVED by the reference; status_mix names them."""
    st = np.array([1, 4, 10, 1], np.int32)  # SOLVED, ALMOST_SOLVED, INSUFFICIENT, SOLVED
    info = np.zeros(4, [("obj_val", "f8")])
    info["obj_val"] = [1.0, 2.0 + 2e-5, 50.0, -3.0]
    res = {"status": st, "info": info}
    ref_solved = np.array([True, True, True, False])
    ref_obj = np.array([1.0 + 1e-9, 2.0, 3.0, -3.0])
    e = bench.obj_errors(res, ref_solved, ref_obj)
    assert e["instances"] == 2
    assert abs(e["max"] - 1e-5) < 1e-12
    assert bench.status_mix(st) == {"SOLVED": 2, "ALMOST_SOLVED": 1,
                                       "INSUFFICIENT_PROGRESS": 1}
