"""Continuous batching (serving): slots admitted while others are mid-solve
must give exactly the results they give when solved in a batch of their own
(every kernel works per instance, so a slot's arithmetic does not depend on
its neighbours or on when it was admitted)."""
import numpy as np
import pytest

from cuclarabel_b200 import BatchSolver, problems

pytestmark = pytest.mark.gpu


def _serve_all(s, schedule, data=None):
    """Admit the slot groups of `schedule` one group per step (while earlier
    groups run), step until everything finished; returns slot -> solution."""
    out, pending = {}, list(schedule)
    running, steps = 0, 0
    while pending or running:
        steps += 1
        assert steps < 1000, "serving did not finish"
        if pending:
            grp = pending.pop(0)
            q = [data[k][0] for k in grp] if data else None
            b = [data[k][1] for k in grp] if data else None
            s.serve_admit(grp, q=q, b=b)
        fin, running = s.serve_step()
        for k, sol in zip(fin, s.serve_collect(fin)):
            out[k] = sol
    return out


def _same(a, b):
    assert a.status == b.status and a.iterations == b.iterations
    assert np.array_equal(a.x, b.x) and np.array_equal(a.z, b.z) and np.array_equal(a.s, b.s)
    assert a.obj_val == b.obj_val


def test_served_results_equal_batch_results(cuda_device):
    pbs = problems.mpc_batch(20, seed0=900)
    ref = BatchSolver(pbs).solve()
    s = BatchSolver(pbs)
    got = _serve_all(s, [[3, 7, 11], [0], [1, 2, 19, 18], [4, 5, 6], list(range(8, 11)),
                         list(range(12, 18))])
    assert sorted(got) == list(range(20))
    for k in range(20):
        _same(got[k], ref[k])


def test_served_new_data_equals_updated_batch(cuda_device):
    rng = np.random.default_rng(3)
    pbs = problems.mpc_batch(12, seed0=950)
    new = {}
    for k, (P, q, A, b, cones) in enumerate(pbs):
        new[k] = (q + 0.1 * rng.standard_normal(len(q)),
                  b + 0.05 * np.abs(rng.standard_normal(len(b))))
    ref_solver = BatchSolver(pbs)
    ref_solver.update_data(q=[new[k][0] for k in range(12)], b=[new[k][1] for k in range(12)])
    ref = ref_solver.solve()
    s = BatchSolver(pbs)
    got = _serve_all(s, [[0, 1, 2, 3], [4, 5], [6, 7, 8, 9, 10, 11]], data=new)
    for k in range(12):
        _same(got[k], ref[k])


def test_slot_reuse_and_errors(cuda_device):
    pbs = problems.mpc_batch(4, seed0=990)
    ref = BatchSolver(pbs).solve()
    s = BatchSolver(pbs)
    s.serve_admit([0, 1])
    with pytest.raises(RuntimeError):
        s.serve_admit([1])          # already admitted
    with pytest.raises(RuntimeError):
        s.serve_admit([2, 2])       # repeated slot
    with pytest.raises(RuntimeError):
        s.serve_admit([2])          # a second admission before a step
    got = {}
    for _ in range(1000):
        fin, running = s.serve_step()
        for k, sol in zip(fin, s.serve_collect(fin)):
            got[k] = sol
        if not running:
            break
    assert sorted(got) == [0, 1]
    # a collected slot is idle again and solves the same way a second time
    s.serve_admit([1, 3])
    for _ in range(1000):
        fin, running = s.serve_step()
        for k, sol in zip(fin, s.serve_collect(fin)):
            got[k] = sol
        if not running:
            break
    assert sorted(got) == [0, 1, 3]
    for k in (0, 1, 3):
        _same(got[k], ref[k])
    # solve! after serving solves every instance again
    again = s.solve()
    for k in range(4):
        _same(again[k], ref[k])


def test_served_supernodal_slots_equal_their_lone_solves(cuda_device):
    """Large slots (configuration-2-like structures on the supernodal
    factorisation, the serving configuration's large requests) admitted
    while another is mid-solve give exactly their lone results: the
    supernodal launches cover only running instances and every reduction
    has a fixed order."""
    pbs = [problems.mixed_socp(0.08, seed=41), problems.mixed_socp(0.1, seed=42),
           problems.mixed_socp(0.09, seed=43)]
    alone = [BatchSolver([pb]).solve()[0] for pb in pbs]
    s = BatchSolver(pbs)
    got = _serve_all(s, [[1], [], [0, 2]])
    for k in range(3):
        _same(got[k], alone[k])
