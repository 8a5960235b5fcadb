"""Request loop for serving (continuous batching) on one GPU.

The reference has no serving loop; this module is the serving pattern of the
benchmark plan: a Poisson stream of solves of different sizes, admitted
while others are on the GPU, with p50/p99 latency beside throughput.

Lanes.  A lane is one resident BatchSolver whose instances are slots
(fixed P / A structure and cones; a request brings new q / b), driven by a
host thread of its own on a CUDA stream of its own, so lanes overlap on the
device and a slow lane (large problems on the supernodal factorisation) does
not hold back a fast one.  Each lane thread runs the slot protocol of
clgpu_serve_admit / clgpu_serve_step / clgpu_serve_collect: requests wait
in per-slot FIFO queues, join at an IPM-step boundary once their slot is
free, run one IPM iteration per step together with every other running
slot, and are collected when they finish.

Cohorts.  Requests whose structure is not resident (new P / A / cones) are
solved by cohorts: the requests waiting when the cohort lane is free are
set up together as one BatchSolver (device setup), admitted when the
budget allows, stepped to completion on the cohort lane's stream and freed.

HBM budget.  Every lane holds the device bytes of its solver in a shared
budget (120 GB in the serving configuration).  A cohort is admitted only
when its estimated bytes fit next to what is held; the estimate is the
bytes per KKT nonzero of the cohorts set up so far (or of the first
resident lane), and the held amount is corrected to the cohort's true bytes
once it exists.

Latency is arrival -> result on the host; all lanes share one clock."""
import collections
import threading
import time

import numpy as np

from .api import BatchSolver


class Budget:
    """Device bytes held against a fixed budget (thread safe)."""

    def __init__(self, total_bytes):
        self.total = int(total_bytes)
        self.held = 0
        self.peak = 0
        self._mu = threading.Lock()

    def try_hold(self, nbytes):
        with self._mu:
            if self.held + nbytes > self.total:
                return False
            self.held += int(nbytes)
            self.peak = max(self.peak, self.held)
            return True

    def hold(self, nbytes):
        with self._mu:
            self.held += int(nbytes)
            self.peak = max(self.peak, self.held)

    def release(self, nbytes):
        with self._mu:
            self.held -= int(nbytes)


def _kkt_nnz(pb):
    P, q, A, b, cones = pb
    return int(P.nnz) + int(A.nnz) + len(q) + len(b)


class _Stats:
    def __init__(self):
        self.lat = []
        self.status = collections.Counter()
        self.iters = []
        self.steps = 0
        self.busy_s = 0.0

    def summary(self, wall):
        lat = np.asarray(self.lat) if self.lat else np.zeros(1)
        out = {"completed": len(self.lat), "solved": self.status.get("SOLVED", 0),
               "status": dict(self.status), "steps": self.steps,
               "solves_per_s": self.status.get("SOLVED", 0) / wall if wall > 0 else 0.0}
        if self.lat:
            out.update(p50_ms=1000 * float(np.percentile(lat, 50)),
                       p99_ms=1000 * float(np.percentile(lat, 99)),
                       iters_mean=float(np.mean(self.iters)))
        return out


class SlotLane:
    """One resident BatchSolver; requests name a slot and carry new q / b.
    `solver` is the BatchSolver (anything with its serve_* and
    device_bytes methods); `kkt_nnz` sizes the budget estimate of cohorts."""

    def __init__(self, name, solver, stream, budget, kkt_nnz=0):
        self.name = name
        self.solver = solver
        self.bytes = self.solver.device_bytes()
        budget.hold(self.bytes)
        self.budget = budget
        self.stream = stream
        self.stats = _Stats()
        self.kkt_nnz = kkt_nnz

    @classmethod
    def build(cls, name, problems, stream, budget, **settings):
        return cls(name, BatchSolver(problems, **settings), stream, budget,
                   sum(_kkt_nnz(pb) for pb in problems))

    def warm(self, slot=0):
        """Serve one request for `slot` to completion before the clock
        starts: the first step of a solver captures its IPM pass (and, on
        the supernodal path, its substitution pass) as CUDA graphs, and no
        other thread may allocate device memory while a capture is open."""
        s = self.solver
        s.serve_admit([slot], stream=self.stream)
        running = 1
        while running:
            fin, running = s.serve_step(self.stream)
            if fin:
                s.serve_collect(fin, self.stream)

    def close(self):
        if self.solver is not None:
            del self.solver
            self.solver = None
            self.budget.release(self.bytes)

    def run(self, t0, arrive, slot, qv, bv, horizon):
        """Serve requests (arrival time, slot, q, b) until all are done or
        `horizon` seconds after t0 pass; returns the number left unfinished."""
        s, st = self.solver, self.stats
        n = len(arrive)
        queues = collections.defaultdict(collections.deque)
        busy = {}
        nxt = running = 0
        while True:
            now = time.perf_counter() - t0
            if now > horizon:
                break
            while nxt < n and arrive[nxt] <= now:
                queues[int(slot[nxt])].append(nxt)
                nxt += 1
            adm, aq, ab = [], [], []
            for k in list(queues):
                if k in busy:
                    continue
                r = queues[k].popleft()
                if not queues[k]:
                    del queues[k]
                adm.append(k)
                aq.append(qv[r])
                ab.append(bv[r])
                busy[k] = r
            if adm:
                s.serve_admit(adm, q=aq, b=ab, stream=self.stream)
                running += len(adm)
            if running:
                a = time.perf_counter()
                fin, running = s.serve_step(self.stream)
                st.steps += 1
                if fin:
                    sols = s.serve_collect(fin, self.stream)
                    done = time.perf_counter() - t0
                    for k, sol in zip(fin, sols):
                        r = busy.pop(k)
                        st.lat.append(done - arrive[r])
                        st.status[sol.status.name] += 1
                        st.iters.append(sol.iterations)
                st.busy_s += time.perf_counter() - a
            elif nxt < n:
                time.sleep(min(0.002, max(0.0, arrive[nxt] - (time.perf_counter() - t0))))
            elif not queues:
                break
        return (n - nxt) + sum(len(v) for v in queues.values()) + len(busy)


class CohortLane:
    """Requests with structures that are not resident: the requests waiting
    when the lane is free are set up as one BatchSolver (at most
    `max_cohort`), admitted under the budget, solved to completion and
    freed."""

    def __init__(self, name, stream, budget, bytes_per_nnz, max_cohort=256, make_solver=None,
                 **settings):
        self.name = name
        self.stream = stream
        self.budget = budget
        self.bytes_per_nnz = float(bytes_per_nnz)
        self.max_cohort = max_cohort
        self.make_solver = make_solver or (lambda pbs: BatchSolver(pbs, **settings))
        self.stats = _Stats()
        self.cohorts = 0
        self.setup_s = 0.0
        self.waited_for_budget = 0

    def run(self, t0, arrive, problems, horizon):
        st = self.stats
        n = len(arrive)
        nxt = 0
        waiting = collections.deque()
        while True:
            now = time.perf_counter() - t0
            if now > horizon:
                break
            while nxt < n and arrive[nxt] <= now:
                waiting.append(nxt)
                nxt += 1
            if not waiting:
                if nxt >= n:
                    break
                time.sleep(min(0.002, max(0.0, arrive[nxt] - (time.perf_counter() - t0))))
                continue
            take = [waiting.popleft() for _ in range(min(self.max_cohort, len(waiting)))]
            pbs = [problems[r] for r in take]
            est = int(self.bytes_per_nnz * sum(_kkt_nnz(pb) for pb in pbs))
            while not self.budget.try_hold(est):
                self.waited_for_budget += 1
                time.sleep(0.001)
                if time.perf_counter() - t0 > horizon:
                    return n - nxt + len(waiting) + len(take)
            a = time.perf_counter()
            solver = self.make_solver(pbs)
            true_bytes = solver.device_bytes()
            self.budget.hold(true_bytes - est)
            self.bytes_per_nnz = max(self.bytes_per_nnz,
                                     true_bytes / max(1, sum(_kkt_nnz(pb) for pb in pbs)))
            self.setup_s += time.perf_counter() - a
            self.cohorts += 1
            solver.serve_admit(list(range(len(pbs))), stream=self.stream)
            running = len(pbs)
            while running:
                fin, running = solver.serve_step(self.stream)
                st.steps += 1
                if fin:
                    sols = solver.serve_collect(fin, self.stream)
                    done = time.perf_counter() - t0
                    for k, sol in zip(fin, sols):
                        st.lat.append(done - arrive[take[k]])
                        st.status[sol.status.name] += 1
                        st.iters.append(sol.iterations)
            del solver
            self.budget.release(true_bytes)
            st.busy_s += time.perf_counter() - a
        return (n - nxt) + len(waiting)


def run_lanes(jobs, horizon, switch_interval=2e-4):
    """Run lane.run(t0, *args) for every (lane, args) in its own thread with
    a common start time; returns (wall seconds, unfinished per lane).  The
    lanes' Python bookkeeping runs under the interpreter lock (the library
    calls release it), so the lock's switch interval is shortened while the
    lanes run: a lane waiting to launch its next step gets the lock within
    `switch_interval` seconds instead of the default 5 ms."""
    import sys
    old = sys.getswitchinterval()
    sys.setswitchinterval(switch_interval)
    try:
        return _run_lanes(jobs, horizon)
    finally:
        sys.setswitchinterval(old)


def _run_lanes(jobs, horizon):
    t0 = time.perf_counter()
    left = [0] * len(jobs)

    def work(i, lane, args):
        left[i] = lane.run(t0, *args, horizon)

    th = [threading.Thread(target=work, args=(i, lane, args)) for i, (lane, args)
          in enumerate(jobs)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return time.perf_counter() - t0, left
