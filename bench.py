"""Benchmark: batched solves/s at 1e-8 for the batched MPC QP/SOCP workload
(4096 independent MPC-style QP/SOCPs, n ~ U{20..400}, m ~ 2n, instance i
seeded with i), compared with the plain one-instance-at-a-time GPU path and
the CPU reference path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--instances B] [--method cudssmixed|cudss]

One step = one solve! of the whole batch (every instance to termination).
`value` is solved instances per second with the problem data resident on
the device (setup excluded, L2 flushed between steps); `e2e` is the same
metric through the public API from host CSC data: Solver(...) setup with its
host->device copies, solve!, and the solutions read back to the host.
Under torchrun each rank solves its own 4096 instances (weak scaling, no
collective on the data path; NCCL only for the barrier and the max-time
reduction).
"""
import argparse
import collections
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def gen_problems(count, seed0):
    from cuclarabel_b200 import problems
    return [problems.mpc_qp(seed0 + i) for i in range(count)]


def algorithmic_bytes_update_scaling(pbs, soc_threshold=5):
    """Bytes of update_scaling per batch launch (NN 32 B/row; SOC 32 B/row +
    8 B/cone, sparse SOC +16 B/row (u, v) + 8 B/cone (d))."""
    total = 0
    for pb in pbs:
        for c in pb[4]:
            t, d, _ = c.spec()
            if t == 1:
                total += 32 * d
            elif t == 2:
                total += 32 * d + 8
                if d > soc_threshold:
                    total += 16 * d + 8
    return total


# ---------------------------------------------------------------- cone kernels
# Cone-kernel roofline workload: the cone types of the large single-problem
# configurations (nonnegative rows and SOC(10) of the mixed QP/SOCP; exp, pow
# and PSD(10) of the exp/pow/PSD LP), one cone-level handle per type (the
# plain B = 1 path through the CompositeConeGPU method table of the C ABI),
# at counts where every vector an operation streams exceeds L2 (126 MB).
CONE_WORKLOAD = {  # name: (type code, dim, cones at scale 1)
    "nn": (1, 16_000_000, 1),
    "soc10": (2, 10, 1_600_000),
    "exp": (3, 3, 4_000_000),
    "pow": (4, 3, 4_000_000),
    "psd10": (5, 10, 400_000),
}
CONE_OPS = ("update_scaling", "mul_Hs", "affine_ds", "combined_ds_shift",
            "ds_from_dz_offset", "step_length")


def cone_op_bytes(op, code, dim, count, soc_threshold=5):
    """Algorithmic bytes of one cone operation over `count` cones of one type:
    every input the operation needs read once and every output written once
    (FP64 values, 8 B).  Per-row state (w, lambda; sparse SOC u, v), per-cone
    state (SOC eta, d; exp/pow gradient, H_dual, Hs and the stored z; PSD
    R, R^-1, lambda) as the kernels of this library keep it."""
    if code == 1:
        per = {"update_scaling": 32, "mul_Hs": 24, "affine_ds": 16,
               "combined_ds_shift": 32, "ds_from_dz_offset": 24, "step_length": 32}
        return per[op] * dim * count
    if code == 2:
        rows = dim * count
        sparse = dim > soc_threshold
        per = {"update_scaling": 32 * rows + 8 * count + ((16 * rows + 8 * count) if sparse else 0),
               "mul_Hs": 24 * rows + 8 * count, "affine_ds": 16 * rows,
               "combined_ds_shift": 32 * rows + 8 * count,
               "ds_from_dz_offset": 40 * rows + 8 * count, "step_length": 32 * rows}
        return per[op]
    if code in (3, 4):
        a = 8 if code == 4 else 0  # the power cone's alpha
        per = {"update_scaling": 240 + a, "mul_Hs": 120, "affine_ds": 48,
               "combined_ds_shift": 192 + a, "ds_from_dz_offset": 48, "step_length": 96 + a}
        return per[op] * count
    n = dim
    t = n * (n + 1) // 2
    per = {"update_scaling": 16 * t + 16 * n * n + 8 * n, "mul_Hs": 8 * n * n + 16 * t,
           "affine_ds": 8 * n + 8 * t, "combined_ds_shift": 24 * t + 16 * n * n,
           "ds_from_dz_offset": 16 * t + 8 * n * n + 8 * n,
           "step_length": 16 * t + 16 * n * n + 8 * n}
    return per[op] * count


def cone_points(code, dim, count, rng, alpha=None):
    """Strictly interior points of `count` cones of one type, concatenated in
    the cone-level row layout, and the power cones' alphas (drawn unless
    given)."""
    if code == 1:
        v = rng.uniform(0.5, 2.0, dim * count)
    elif code == 2:
        tail = rng.standard_normal((count, dim - 1))
        head = 1.0 + np.linalg.norm(tail, axis=1) * rng.uniform(1.05, 2.0, count)
        v = np.concatenate([head[:, None], tail], axis=1).ravel()
    elif code == 3:
        base = np.array([-1.051383945322714, 0.556409619469370, 1.258967884768947])
        v = (base[None, :] * rng.uniform(0.5, 2.0, (count, 1))
             + rng.normal(0, 0.02, (count, 3))).ravel()
    elif code == 4:
        if alpha is None:
            alpha = rng.uniform(0.2, 0.8, count)
        v = np.stack([np.sqrt(1 + alpha), np.sqrt(2 - alpha), np.zeros(count)], axis=1)
        v = v * rng.uniform(0.5, 2.0, (count, 1))
        v[:, 2] = rng.normal(0, 0.1, count)
        v = v.ravel()
    else:
        n = dim
        E = rng.standard_normal((count, n, n)) * 0.1
        M = np.eye(n)[None] + (E + E.transpose(0, 2, 1)) / 2
        ii, jj = [], []
        for j in range(n):
            for i in range(j + 1):
                ii.append(i)
                jj.append(j)
        ii, jj = np.array(ii), np.array(jj)
        scale = np.where(ii == jj, 1.0, np.sqrt(2.0))
        v = (M[:, ii, jj] * scale[None, :]).ravel()
    return v, alpha


def cone_kernel_roofline(hbm, scale=1.0, reps=5, seed=7):
    """Per-kernel device time and HBM throughput of every per-iteration cone
    operation on the cone roofline workload (CUDA events around each
    operation's kernels inside the library, median of `reps` after warm-up,
    L2 flushed before each timed call)."""
    import torch
    from cuclarabel_b200 import _lib
    L = _lib.load()
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    rng = np.random.default_rng(seed)
    out = {}
    for name, (code, dim, count) in CONE_WORKLOAD.items():
        if code == 1:
            dim = max(1, int(dim * scale))
        else:
            count = max(1, int(count * scale))
        types = np.full(count, code, np.int32)
        dims = np.full(count, dim, np.int32)
        s_h, alpha = cone_points(code, dim, count, rng)
        z_h, _ = cone_points(code, dim, count, rng, alpha)
        params = np.ascontiguousarray(alpha if alpha is not None else np.zeros(count),
                                      np.float64)
        h = ctypes.c_void_p()
        rc = L.clgpu_cones_create(count, types.ctypes.data_as(_lib.ip),
                                  dims.ctypes.data_as(_lib.ip), params.ctypes.data_as(_lib.dp),
                                  5, ctypes.byref(h))
        assert rc == 0, (name, rc)
        try:
            assert L.clgpu_cones_set_profiling(h, 1) == 0
            m = L.clgpu_cones_numel(h)

            def dev(a):
                return torch.tensor(np.asarray(a, np.float64), device="cuda")

            s, z = dev(s_h), dev(z_h)
            dz = dev(0.05 * rng.standard_normal(m))
            ds = dev(0.05 * rng.standard_normal(m))
            x = dev(rng.standard_normal(m))
            y = torch.empty(m, dtype=torch.float64, device="cuda")

            def P(t):
                return ctypes.c_void_p(t.data_ptr())

            a_out = ctypes.c_double()
            calls = {
                "update_scaling": lambda: L.clgpu_update_scaling(h, P(s), P(z), 1.0, 0, sh),
                "mul_Hs": lambda: L.clgpu_mul_Hs(h, P(y), P(x), sh),
                "affine_ds": lambda: L.clgpu_affine_ds(h, P(y), P(s), sh),
                "combined_ds_shift": lambda: L.clgpu_combined_ds_shift(
                    h, P(y), P(dz), P(ds), P(z), 0.1, sh),
                "ds_from_dz_offset": lambda: L.clgpu_ds_from_dz_offset(h, P(y), P(ds), P(z), sh),
                "step_length": lambda: L.clgpu_step_length(
                    h, P(dz), P(ds), P(z), P(s), 1.0, 0.99, 0.8, 1e-4, ctypes.byref(a_out), sh),
            }
            nb, sv = ctypes.c_int(), (ctypes.c_int * 6)()
            L.clgpu_cones_get_launch_shapes(h, ctypes.byref(nb), sv)
            shapes = {"nn_block": nb.value,
                      "soc": ["groups" if x == 0 else "tiles%d" % (32 << (x - 1)) for x in sv]}
            res = {}
            for op in CONE_OPS:
                fn = calls[op]
                for _ in range(1 if reps <= 1 else 2):
                    rc = fn()
                    assert rc == 0, (name, op, rc)
                ts = []
                for _ in range(reps):
                    flush.add_(1.0)
                    torch.cuda.synchronize()
                    rc = fn()
                    assert rc == 0, (name, op, rc)
                    ms = ctypes.c_double()
                    L.clgpu_cones_last_kernel_ms(h, ctypes.byref(ms))
                    ts.append(ms.value)
                ms = float(np.median(ts))
                by = cone_op_bytes(op, code, dim, count)
                gbs = by / (ms / 1e3) / 1e9 if ms > 0 else 0.0
                res[op] = {"us": round(1000 * ms, 2), "bytes": int(by),
                           "GB/s": round(gbs, 1), "frac": round(gbs / hbm, 3)}
            out[name] = {"cones": count, "dim": dim, "rows": m, "ops": res,
                         "launch_shapes": shapes if code in (1, 2) else None}
            del s, z, dz, ds, x, y
        finally:
            L.clgpu_cones_destroy(h)
    del flush
    torch.cuda.synchronize()
    return out


def problem_bytes(pbs):
    b = 0
    for P, q, A, bb, c in pbs:
        b += P.nnz * 12 + (P.shape[1] + 1) * 4 + A.nnz * 12 + (A.shape[1] + 1) * 4
        b += q.nbytes + bb.nbytes + len(c) * 12
    return b


def _ref_worker(w, nworkers, count, conn):
    """One CPU worker: owns instances w, w + nworkers, ... of the workload and
    sets each up once (Solver(...): equilibration, KKT assembly, ordering,
    symbolic factorisation).  On "go" it runs solve! on its slice; on "cold"
    it solves its slice from scratch (setup included).  Reports (solved,
    seconds)."""
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    import oracle
    from cuclarabel_b200 import problems
    mine = [problems.mpc_qp(i) for i in range(w, count, nworkers)]
    objs = [oracle.SolverObject(*pb, gpu_equilibration=1) for pb in mine]
    conn.send("ready")
    last = []
    while True:
        msg = conn.recv()
        if msg == "objs":  # (SOLVED, objective) of every instance of the last "go"
            conn.send(last)
            continue
        if msg not in ("go", "cold"):
            break
        t0 = time.perf_counter()
        if msg == "go":
            res = [o.run() for o in objs]
            solved = sum(1 for r in res if r["status_name"] == "SOLVED")
            last = [(r["status_name"] == "SOLVED", r["obj_val"]) for r in res]
        else:
            solved = sum(1 for pb in mine
                         if oracle.solve(*pb, gpu_equilibration=1)["status_name"] == "SOLVED")
        conn.send((solved, time.perf_counter() - t0))


class RefPool:
    """The CPU reference path (the oracle's restatement of the reference's
    CPU solver) over all host cores, one process per core, each owning a
    fixed slice of the workload so that problem generation stays outside the
    timed region."""

    def __init__(self, count):
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        self.cores = os.cpu_count() or 1
        self.count = count
        self.conns, self.procs = [], []
        for w in range(self.cores):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_ref_worker, args=(w, self.cores, count, b), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        for c in self.conns:
            assert c.recv() == "ready"

    def step(self, cold=False):
        t0 = time.perf_counter()
        for c in self.conns:
            c.send("cold" if cold else "go")
        solved = 0
        for c in self.conns:
            s, _ = c.recv()
            solved += s
        return solved, time.perf_counter() - t0

    def objectives(self):
        """(SOLVED mask, objective) per instance of the last step."""
        solved = np.zeros(self.count, bool)
        obj = np.full(self.count, np.nan)
        for w, c in enumerate(self.conns):
            c.send("objs")
            for k, (ok, ov) in enumerate(c.recv()):
                solved[w + k * self.cores] = ok
                obj[w + k * self.cores] = ov
        return solved, obj

    def close(self):
        for c in self.conns:
            c.send("stop")
        for p in self.procs:
            p.join(timeout=10)


def run_reference(args, rank, world):
    """`--impl reference`: the reference's CPU algorithm (the oracle port) on
    the host cores for the same workload, metric and unit as the GPU arm.
    Under torchrun only rank 0 runs; the other ranks exit without work."""
    if rank != 0:
        return
    B = args.instances
    pool = RefPool(B)
    times, solved = [], 0
    for step in range(args.warmup + args.steps):
        s, dt = pool.step()
        if step >= args.warmup:
            times.append(dt)
            solved += s
    cold_solved, cold_dt = pool.step(cold=True)
    pool.close()
    total = sum(times)
    val = solved / total
    line = {
        "metric": METRIC, "value": val, "unit": "solves/s", "impl": "reference",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64, MPC batch shapes)",
        "config": workload_config(B, args.method),
        "cpu_baseline": {"value": val, "unit": "solves/s", "cores": pool.cores, "kind": "port",
                         "sample": "the full %d-instance workload per step: solve! of every "
                                   "instance on solvers set up beforehand, one process per "
                                   "core, each owning a fixed slice" % B},
        "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "cold": {"value": cold_solved / cold_dt, "unit": "solves/s",
                 "note": "one pass with setup included (Solver(...) + solve! per instance)"},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(count):
    """The CPU reference path over `count` instances (the GPU arm's
    cpu_baseline field): solve! on solvers set up beforehand, three passes
    (~2 ms of CPU per instance and pass)."""
    pool = RefPool(count)
    solved, dt = 0, 0.0
    for _ in range(3):
        s_, d_ = pool.step()
        solved += s_
        dt += d_
    checker = pool.objectives()
    pool.close()
    return {"value": solved / dt, "unit": "solves/s", "cores": pool.cores, "kind": "port",
            "sample": "%d MPC QP/SOCP instances (the workload's first %d) x 3 passes of solve! "
                      "on solvers set up beforehand, one process per core, %.1f s wall"
                      % (count, count, dt)}, checker


METRIC = "solves/s at 1e-8 (batched MPC QP/SOCP)"


def pinned_stats():
    """Counters of the library's page-locked host pool (reused, new, bytes,
    failed)."""
    import ctypes
    from cuclarabel_b200 import _lib
    out = (ctypes.c_longlong * 4)()
    _lib.load().clgpu_debug_pinned_stats(out)
    return list(out)


def status_mix(status):
    from cuclarabel_b200 import SolverStatus
    out = {}
    for v in status:
        nm = SolverStatus(int(v)).name
        out[nm] = out.get(nm, 0) + 1
    return out


def obj_errors(res, ref_solved, ref_obj):
    """Relative objective errors of the instances `res` converged on (SOLVED
    or ALMOST_SOLVED) among those the reference run SOLVED."""
    from cuclarabel_b200 import SolverStatus
    conv = (res["status"] == int(SolverStatus.SOLVED)) | \
           (res["status"] == int(SolverStatus.ALMOST_SOLVED))
    n = min(len(conv), len(ref_solved))
    both = conv[:n] & np.asarray(ref_solved[:n], bool)
    rel = np.abs(res["info"]["obj_val"][:n] - ref_obj[:n]) / np.maximum(1.0, np.abs(ref_obj[:n]))
    return {"instances": int(both.sum()),
            "max": float(rel[both].max()) if both.any() else None,
            "median": float(np.median(rel[both])) if both.any() else None}


def workload_config(B, method):
    return {"workload": "%d MPC-style QP/SOCPs per GPU, n~U{20..400}, m~2n, 5-20 SOC(3..8)"
                        % B, "instances_per_gpu": B, "method": method}


def ncu_traffic(summary):
    """DRAM bytes (read + write) of one launch from a committed ncu summary
    under profiles/ (its dram_bytes_per_launch line), or None."""
    p = os.path.join(ROOT, "profiles", summary)
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def fp64_gemm_peak():
    """cuBLAS FP64 GEMM throughput on this GPU (torch.matmul, 8192^3, best of
    10 after warm-up): the denominator of the FP64 tensor-core roofline."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(3):
        a @ b
    torch.cuda.synchronize()
    best = None
    for _ in range(10):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1)
        best = t if best is None else min(best, t)
    del a, b
    return 2.0 * n ** 3 / (best / 1000.0) / 1e12


def _oracle_sample_worker(which, scale, conn):
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    import oracle
    from cuclarabel_b200 import problems
    pb = problems.mixed_socp(scale) if which == 2 else problems.exp_pow_psd(scale)
    obj = oracle.SolverObject(*pb, gpu_equilibration=1)
    t0 = time.perf_counter()
    r = obj.run()
    conn.send((r["status_name"], r["iterations"], time.perf_counter() - t0))


def large_single(which, scale, method, sh, fp64_peak, cpu_scale):
    """One large single problem (configuration 2: mixed SOCP, n = 20000,
    m = 60000; configuration 3: exp/pow/PSD LP, n = 30000, m = 96000, at
    `scale`) on the supernodal LDL^T: setup, a profiled solve for the
    per-kernel breakdown (which also warms up), a solve timed with CUDA
    events (L2 flushed before), and the end-to-end pass (new values from
    pinned host memory + solve! + solution read back)."""
    import torch
    from cuclarabel_b200 import Solver, SolverStatus, problems
    from cuclarabel_b200.api import _as_csc
    pb = problems.mixed_socp(scale) if which == 2 else problems.exp_pow_psd(scale)
    t0 = time.perf_counter()
    s = Solver(*pb, direct_solve_method=method)
    setup_s = time.perf_counter() - t0
    s.set_profiling(True)
    s.solve(sh)
    prof = s.profile()
    s.set_profiling(False)
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device="cuda")
    flush.add_(1.0)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.ExternalStream(sh)
    e0.record(stream)
    s.solve_only(sh)
    e1.record(stream)
    torch.cuda.synchronize()
    dev_s = e0.elapsed_time(e1) / 1000.0
    sol = s.solutions()[0]
    sn = prof.get("supernodal", {})
    upd = sn.get("update", {"ms": 0.0, "flops": 0.0, "launches": 0})
    fact_fl = sum(v["flops"] for v in sn.values())
    fact_ms = sum(sn[k]["ms"] for k in ("small_fronts", "assemble", "diag", "trsm", "update")
                  if k in sn)
    solve_ms = sum(v["ms"] for k, v in sn.items() if k.startswith(("fwd", "bwd")))
    ach = upd["flops"] / (upd["ms"] / 1000.0) / 1e12 if upd["ms"] > 0 else 0.0
    # end to end: new P, q, A, b values from pinned host memory, solve!, x/s/z back
    P, q, A, b, _ = pb
    vals = [_as_csc(P, P.shape).data, np.asarray(q, np.float64),
            _as_csc(A, A.shape).data, np.asarray(b, np.float64)]
    pinned = []
    for v in vals:
        t = torch.empty(len(v), dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = v
        pinned.append(t.numpy())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.update_data(P=pinned[0], q=pinned[1], A=pinned[2], b=pinned[3], stream=sh)
    s.solve_only(sh)
    res = s.results()
    e2e_s = time.perf_counter() - t0
    ok = res["status"][0] == int(SolverStatus.SOLVED)
    out = {
        "workload": ("config 2: mixed-cone QP/SOCP n=%d, m=%d (2000 zero, 28000 nonneg, "
                     "3000 SOC(10) at scale 1)" if which == 2 else
                     "config 3: exp/pow/PSD LP n=%d, m=%d (20000 exp, 5000 pow, 200 PSD(10), "
                     "10000 nonneg at scale 1)") % (A.shape[1], A.shape[0]),
        "scale": scale, "method": method,
        "value": (1.0 / dev_s) if sol.status == SolverStatus.SOLVED else 0.0,
        "solve_rate_any_status": 1.0 / dev_s,
        "unit": "solves/s", "solve_s": dev_s, "setup_s": setup_s,
        "status": sol.status.name, "iterations": sol.iterations, "obj_val": sol.obj_val,
        "device_bytes": s.device_bytes(),
        "e2e": {"value": (1.0 / e2e_s) if ok else 0.0, "unit": "solves/s",
                "h2d_bytes_per_step": int(sum(v.nbytes for v in vals)),
                "d2h_bytes_per_step": int(8 * (A.shape[1] + 2 * A.shape[0])),
                "note": "update_data! of P, q, A, b from pinned host memory + solve! + x, s, "
                        "z read back; solver set up beforehand"},
        "factor": {"ms_per_solve": fact_ms, "flops_per_solve": fact_fl,
                   "tflops": fact_fl / (fact_ms / 1000.0) / 1e12 if fact_ms > 0 else 0.0,
                   "factorisations": sn.get("diag", {}).get("launches", 0)},
        "solves_ms_per_solve": solve_ms,
        "kernels": {k: {"ms": round(v["ms"], 3), "launches": v["launches"]}
                    for k, v in sn.items() if v["launches"]},
        "roofline": {"bound": "tensor", "kernel": "k_sn_update_f64 (trailing update of "
                     "the blocked fronts, m8n8k4 FP64 DMMA)" if method == "cudss" else
                     "k_sn_update_f32 (trailing update, FP32 FMA)",
                     "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": ach / fp64_peak if fp64_peak else None,
                     "peak_kind": "measured: cuBLAS FP64 GEMM 8192^3 on this GPU in this run",
                     "flops_per_launch": upd["flops"] / max(upd["launches"], 1),
                     "avg_launch_ms": upd["ms"] / max(upd["launches"], 1),
                     "launches": upd["launches"], "traffic": None},
    }
    del s
    if cpu_scale > 0:
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        a, b_ = ctx.Pipe()
        p = ctx.Process(target=_oracle_sample_worker, args=(which, cpu_scale, b_), daemon=True)
        p.start()
        st_, it_, dt_ = a.recv()
        p.join(timeout=10)
        out["cpu_baseline"] = {
            "value": (1.0 / dt_) if st_ == "SOLVED" else 0.0, "unit": "solves/s", "cores": 1,
            "kind": "port", "status": st_, "iterations": it_, "seconds": dt_,
            "sample": "the same family at scale %.3f (the oracle's scalar LDL^T of the full "
                      "size does not finish in minutes), solve! on a solver set up "
                      "beforehand, one core" % cpu_scale}
    return out


def rank_seed0(rank, instances):
    """First instance seed of a rank: rank r owns instances [r B, (r+1) B),
    so ranks share no instance (weak scaling, no data-path collective)."""
    return rank * instances


def aggregate_over_ranks(elapsed, solved, dist, device):
    """Whole-job figures: the slowest rank's time and every rank's solves
    (the only collectives of the multi-GPU run)."""
    if dist is None:
        return elapsed, solved
    import torch
    t = torch.tensor([elapsed, float(solved)], device=device, dtype=torch.float64)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return tmax[0].item(), int(round(tsum[1].item()))


def _b_noise(rng, cones, m):
    """A request's change of b: +0.02 |N(0,1)| on the inequality rows (the
    slack grows, so the problem stays feasible); equality (zero-cone) rows
    keep their values, since an empty equality row must keep b = 0."""
    from cuclarabel_b200.api import ZeroConeT
    mask = np.ones(m)
    row = 0
    for c in cones:
        d = c.nvars()
        if isinstance(c, ZeroConeT):
            mask[row:row + d] = 0.0
        row += d
    return 0.02 * np.abs(rng.standard_normal(m)) * mask


# scales of the large (configuration-2-like) request structures of the
# serving configuration: n = 20000 * scale spans 2000..20000
SERVE_LARGE_SCALES = (0.1, 0.2, 0.35, 0.5, 0.75, 1.0)


def serve_config5(pbs, lam, seconds, seed, method, budget_gb, new_frac, large_frac, grace,
                  plain_small_pool):
    """The serving configuration under a Poisson stream of `lam` requests/s
    for `seconds`: a `large_frac` share of configuration-2-like requests
    (n from 2000 to 20000, resident structures on the supernodal path, new
    q / b), a `new_frac` share of MPC requests with structures that are not
    resident (set up in cohorts under the HBM budget), the rest MPC requests
    for the resident batch's structures (new q / b).  The served arm runs
    the three lanes of cuclarabel_b200.serving concurrently; the plain arm
    then serves the same arrivals one request at a time (FIFO) on
    single-instance solvers.  Both arms stop at `seconds + grace`; requests
    still open then are reported as unfinished."""
    import torch
    from cuclarabel_b200 import Solver, problems
    from cuclarabel_b200 import serving
    rng = np.random.default_rng(seed)
    B = len(pbs)
    n = int(rng.poisson(lam * seconds))
    arrive = np.sort(rng.uniform(0.0, seconds, n))
    u = rng.uniform(size=n)
    cls = np.where(u < large_frac, 2, np.where(u < large_frac + new_frac, 1, 0))
    large_pbs = [problems.mixed_socp(sc, seed=40 + k) for k, sc in enumerate(SERVE_LARGE_SCALES)]
    which = np.where(cls == 2, rng.integers(0, len(large_pbs), n), rng.integers(0, B, n))
    qv, bv, newp = [None] * n, [None] * n, {}
    for r in range(n):
        if cls[r] == 1:
            newp[r] = problems.mpc_qp(1000000 + r)
            continue
        P, q, A, b, cones = (large_pbs if cls[r] == 2 else pbs)[which[r]]
        qv[r] = q + 0.05 * rng.standard_normal(len(q))
        bv[r] = b + _b_noise(rng, cones, len(b))
    idx = [np.nonzero(cls == c)[0] for c in range(3)]
    horizon = seconds + grace

    # ---- served arm: three lanes, one thread and stream each
    budget = serving.Budget(budget_gb * 1e9)
    # the MPC lanes' streams take the highest priority, the large lane's the
    # lowest: the block scheduler then fills free SMs with MPC work first,
    # so the large lane's long kernels do not set the MPC requests' latency
    lo, hi = torch.cuda.Stream.priority_range() if hasattr(torch.cuda.Stream,
                                                           "priority_range") else (0, -1)
    streams = [torch.cuda.Stream(priority=hi), torch.cuda.Stream(priority=lo),
               torch.cuda.Stream(priority=hi)]
    t_setup = time.perf_counter()
    small = serving.SlotLane.build("resident MPC", pbs, streams[0].cuda_stream, budget,
                                   direct_solve_method=method)
    large = serving.SlotLane.build("resident config-2-like", large_pbs, streams[1].cuda_stream,
                                   budget, direct_solve_method=method)
    # cohorts are set up while the other lanes run: no launch-shape timing
    # (its L2 flushes and timed launches would disturb them)
    cohort = serving.CohortLane("new-structure MPC", streams[2].cuda_stream, budget,
                                bytes_per_nnz=small.bytes / max(small.kkt_nnz, 1),
                                direct_solve_method=method, autotune=False,
                                setup_threads=2)
    small.warm(0)
    large.warm(0)  # the smallest configuration-2-like structure
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    jobs = [(small, (arrive[idx[0]], which[idx[0]], [qv[r] for r in idx[0]],
                     [bv[r] for r in idx[0]])),
            (large, (arrive[idx[2]], which[idx[2]], [qv[r] for r in idx[2]],
                     [bv[r] for r in idx[2]])),
            (cohort, (arrive[idx[1]], [newp[r] for r in idx[1]]))]
    wall, left = serving.run_lanes(jobs, horizon)
    lanes = {}
    all_lat, solved = [], 0
    for (lane, _), lf in zip(jobs, left):
        d = lane.stats.summary(wall)
        d["requests"] = int(len(_[0]))
        d["unfinished"] = int(lf)
        lanes[lane.name] = d
        all_lat += lane.stats.lat
        solved += d["solved"]
    served = {"lambda_per_s": lam, "seconds": seconds, "grace_s": grace, "requests": n,
              "completed": len(all_lat), "unfinished": int(sum(left)),
              "value": solved / wall, "unit": "solves/s", "wall_s": wall,
              "p50_ms": 1000 * float(np.percentile(all_lat, 50)) if all_lat else None,
              "p99_ms": 1000 * float(np.percentile(all_lat, 99)) if all_lat else None,
              "lanes": lanes, "setup_s": setup_s,
              "hbm_budget_gb": budget_gb, "hbm_peak_held_gb": budget.peak / 1e9,
              "cohorts": cohort.cohorts, "cohort_setup_s": cohort.setup_s,
              "cohort_budget_waits": cohort.waited_for_budget,
              "mix": {"resident_mpc": int(len(idx[0])), "new_structure_mpc": int(len(idx[1])),
                      "config2_like": int(len(idx[2]))}}
    small.close()
    large.close()
    del small, large, cohort
    torch.cuda.synchronize()

    # ---- plain arm: the same arrivals, one request at a time
    pool = [Solver(*pbs[k], direct_solve_method=method) for k in range(min(plain_small_pool, B))]
    lsol = [Solver(*pb, direct_solve_method=method) for pb in large_pbs]
    solvers, pw = [], np.empty(n, np.int64)
    for r in range(n):
        if cls[r] == 0:
            pw[r] = which[r] % len(pool)
        elif cls[r] == 2:
            pw[r] = len(pool) + which[r]
        else:
            pw[r] = -1
    solvers = pool + lsol
    lat, status = [], collections.Counter()
    prng = np.random.default_rng(seed + 1)
    t0 = time.perf_counter()
    unfinished = 0
    for r in range(n):
        now = time.perf_counter() - t0
        if now > horizon:
            unfinished = n - r
            break
        if arrive[r] > now:
            time.sleep(arrive[r] - now)
        if pw[r] >= 0:
            s_ = solvers[pw[r]]
            if cls[r] == 0:  # new q / b for the pool structure that serves it
                _, q0, _, b0, c0_ = pbs[pw[r]]
                s_.update_data(q=q0 + 0.05 * prng.standard_normal(len(q0)),
                               b=b0 + _b_noise(prng, c0_, len(b0)))
            else:
                s_.update_data(q=qv[r], b=bv[r])
            sol = s_.solve()
        else:
            s_ = Solver(*newp[r], direct_solve_method=method)
            sol = s_.solve()
            del s_
        lat.append(time.perf_counter() - t0 - arrive[r])
        status[sol.status.name] += 1
    pwall = time.perf_counter() - t0
    plain = {"requests": n, "completed": len(lat), "unfinished": unfinished,
             "value": status.get("SOLVED", 0) / pwall, "unit": "solves/s", "wall_s": pwall,
             "p50_ms": 1000 * float(np.percentile(lat, 50)) if lat else None,
             "p99_ms": 1000 * float(np.percentile(lat, 99)) if lat else None,
             "status": dict(status),
             "note": "run, not replayed: the same arrivals served one at a time, first come "
                     "first served, on single-instance solvers (resident MPC requests on a pool "
                     "of %d solvers, slot mod pool; config-2-like requests on one solver per "
                     "structure; new structures set up per request); requests still queued "
                     "at the horizon are unfinished and not in p50/p99" % len(pool)}
    del pool, lsol, solvers
    torch.cuda.synchronize()
    served["plain_under_same_load"] = plain
    return served


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--method", default="cudss")
    ap.add_argument("--plain-sample", type=int, default=48)
    ap.add_argument("--ref-sample", type=int, default=4096)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="length of the served (continuous batching) run; 0 skips it")
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--serve-new-frac", type=float, default=0.05,
                    help="share of MPC requests whose structure is not resident")
    ap.add_argument("--serve-large-frac", type=float, default=0.05,
                    help="share of configuration-2-like requests (n 2000..20000)")
    ap.add_argument("--serve-grace", type=float, default=10.0,
                    help="seconds after the last arrival before both arms stop")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving configuration and print its JSON")
    ap.add_argument("--plain-pool", type=int, default=256,
                    help="single-instance solvers of the plain arm for resident MPC structures")
    ap.add_argument("--cone-scale", type=float, default=1.0,
                    help="size of the cone-kernel roofline workload (1.0: every streamed "
                         "vector larger than L2); 0 skips it")
    ap.add_argument("--cone-reps", type=int, default=5,
                    help="timed calls per cone operation (median reported)")
    ap.add_argument("--cone-kernels-only", action="store_true",
                    help="run only the cone-kernel roofline workload and print its JSON")
    ap.add_argument("--large-scale", type=float, default=1.0,
                    help="scale of the large single problems (configurations 2 and 3) run "
                         "on the supernodal factorisation; 0 skips them")
    ap.add_argument("--large-cpu-scale", type=float, default=0.05,
                    help="scale of the CPU oracle's sample of configurations 2 and 3")
    ap.add_argument("--large-which", type=int, default=0, choices=(0, 2, 3),
                    help="with --large-only: configuration 2 or 3 only (0: both)")
    ap.add_argument("--large-only", action="store_true",
                    help="run only configurations 2 and 3 and print their JSON")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    if args.cone_kernels_only:
        peaks, _ = load_peaks()
        hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
        print(json.dumps({"cone_kernels": cone_kernel_roofline(hbm, args.cone_scale,
                                                               args.cone_reps),
                          "peak_gbs": hbm}), flush=True)
        return
    if args.large_only:
        from cuclarabel_b200 import problems as _p  # noqa: F401
        st_ = torch.cuda.Stream()
        pk = fp64_gemm_peak()
        out = {"fp64_gemm_tflops": pk}
        for which in ((2, 3) if args.large_which == 0 else (args.large_which,)):
            out["config%d" % which] = large_single(which, args.large_scale, args.method,
                                                   st_.cuda_stream, pk,
                                                   0 if args.no_cpu else args.large_cpu_scale)
        print(json.dumps(out), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from cuclarabel_b200 import BatchSolver, Solver, SolverStatus, _lib

    B = args.instances
    seed0 = rank_seed0(rank, B)
    pbs = gen_problems(B, seed0)
    if args.serve_only:
        print(json.dumps({"served": serve_config5(
            pbs, args.serve_rate, args.serve_seconds, 12345 + rank, args.method,
            args.serve_budget_gb, args.serve_new_frac, args.serve_large_frac,
            args.serve_grace, args.plain_pool)}), flush=True)
        return
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    solver = BatchSolver(pbs, direct_solve_method=args.method)
    dev_bytes = solver.device_bytes()
    launch_shapes = solver.launch_shapes()  # chosen by the setup autotuner
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device="cuda")

    def flush_l2():
        flush.add_(1.0)
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        solver.solve(sh)
    # profiled (untimed) pass for the phase breakdown
    solver.set_profiling(True)
    sols = solver.solve(sh)
    prof = solver.profile()
    solver.set_profiling(False)
    launches_per_solve = solver.launch_count()

    sampler = ClockSampler(local)
    times = []
    solved_total = 0
    sampler.start()
    for _ in range(args.steps):
        flush_l2()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.solve_only(sh)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1000.0)
        res = solver.results()
        solved_total += int(np.sum(res["status"] == int(SolverStatus.SOLVED)))
    sols = solver.solutions()
    clocks = sampler.stop()
    elapsed, solved_total = aggregate_over_ranks(sum(times), solved_total, dist, "cuda")
    value = solved_total / elapsed
    n_solved_last = sum(1 for s in sols if s.status == SolverStatus.SOLVED)
    status_counts = {}
    for s in sols:
        status_counts[s.status.name] = status_counts.get(s.status.name, 0) + 1
    iters = [s.iterations for s in sols]

    # ---- e2e through the public API with host buffers: every step copies the
    # whole batch's problem values from pinned host memory (update_data!,
    # the reference's data-update path on solvers set up beforehand), solves,
    # and reads every solution and info record back to the host
    from cuclarabel_b200.api import _as_csc
    Pv = np.concatenate([_as_csc(pb[0], pb[0].shape).data for pb in pbs])
    Av = np.concatenate([_as_csc(pb[2], pb[2].shape).data for pb in pbs])
    qv = np.concatenate([np.asarray(pb[1], np.float64) for pb in pbs])
    bv = np.concatenate([np.asarray(pb[3], np.float64) for pb in pbs])
    pinned = []
    for v in (Pv, qv, Av, bv):
        t = torch.empty(len(v), dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = v
        pinned.append(t)
    Pp_, qp_, Ap_, bp_ = [t.numpy() for t in pinned]
    s2 = BatchSolver(pbs, direct_solve_method=args.method)  # setup outside the timed region
    res_buf = None
    for _ in range(2):
        s2.update_data(P=Pp_, q=qp_, A=Ap_, b=bp_, stream=sh)
        s2.solve_only(sh)
        res_buf = s2.results(res_buf, view=True)
    e2e_steps = max(1, args.steps)
    e2e_t = 0.0
    e2e_solved = 0
    for _ in range(e2e_steps):
        flush_l2()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2.update_data(P=Pp_, q=qp_, A=Ap_, b=bp_, stream=sh)
        s2.solve_only(sh)
        res = s2.results(res_buf, view=True)  # x, s, z read from the pinned staging
        e2e_t += time.perf_counter() - t0
        e2e_solved += int(np.sum(res["status"] == int(SolverStatus.SOLVED)))
    h2d = 8 * (len(Pv) + len(qv) + len(Av) + len(bv))
    d2h = 8 * (s2.nx + 2 * s2.mz) + B * ctypes.sizeof(_lib.ClgpuInfo)
    del s2, res, res_buf  # the result views hold the solver (and its staging) alive
    e2e_t, e2e_solved = aggregate_over_ranks(e2e_t, e2e_solved, dist, "cuda")
    e2e_val = e2e_solved / e2e_t
    # cold path for reference: Solver(...) setup from host CSC data + solve +
    # solutions, one pass
    torch.cuda.synchronize()
    pool0 = pinned_stats()
    t0 = time.perf_counter()
    s3 = BatchSolver(pbs, direct_solve_method=args.method)
    t1 = time.perf_counter()
    pool1 = pinned_stats()
    s3.solve_only(sh)
    t2 = time.perf_counter()
    res3 = s3.results()
    cold_t = time.perf_counter() - t0
    cold = {"value": float(np.sum(res3["status"] == int(SolverStatus.SOLVED))) / cold_t,
            "unit": "solves/s", "setup_s": t1 - t0, "solve_s": t2 - t1,
            "results_s": cold_t - (t2 - t0),
            "pinned_pool": {"reused": pool1[0] - pool0[0], "new": pool1[1] - pool0[1],
                            "new_mb": (pool1[2] - pool0[2]) / 2**20,
                            "failed": pool1[3] - pool0[3], "held_mb": pool1[2] / 2**20},
            "note": "one pass: Solver(...) setup from host CSC data (equilibration, "
                    "ordering, symbolic LDL) + solve! + results"}
    del s3

    # ---- mixed precision: direct_solve_method = :cudssmixed (FP32
    # elimination, FP32 factor, FP64 refinement) and mixed_f64elim (FP64
    # elimination, FP32 factor, FP64 refinement); same batch, timed the same
    # way, each objective against the FP64 run's (and, once the CPU leg has
    # run, against the oracle's)
    mixed = None
    mixed_res = {}
    if rank == 0 and args.method == "cudss":
        res64 = solver.results()
        mixed = {}
        for meth in ("cudssmixed", "mixed_f64elim"):
            sm_ = BatchSolver(pbs, direct_solve_method=meth)
            sm_.solve_only(sh)
            mt, msolved = 0.0, 0
            for _ in range(3):
                flush_l2()
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sm_.solve_only(sh)
                e1.record(stream)
                torch.cuda.synchronize()
                mt += e0.elapsed_time(e1) / 1000.0
                r32 = sm_.results()
                msolved += int(np.sum(r32["status"] == int(SolverStatus.SOLVED)))
            del sm_
            mixed_res[meth] = r32
            mixed[meth] = {"value": msolved / mt, "unit": "solves/s",
                           "ms_per_step": 1000 * mt / 3, "status": status_mix(r32["status"]),
                           "obj_rel_err_vs_fp64": obj_errors(
                               r32, res64["status"] == int(SolverStatus.SOLVED),
                               res64["info"]["obj_val"]),
                           "note": "SOLVED at 1e-8 per second; objectives of instances "
                                   "converged (SOLVED or ALMOST_SOLVED) against those the "
                                   "reference solves"}

    # ---- plain path: one instance at a time on the same GPU (FP64, B = 1)
    plain = None
    if rank == 0 and args.plain_sample > 0:
        ps = [Solver(*pbs[i]) for i in range(args.plain_sample)]
        for s in ps[:3]:
            s.solve(sh)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lat = []
        nsol = 0
        for s in ps:
            a = time.perf_counter()
            r = s.solve(sh)
            lat.append(time.perf_counter() - a)
            nsol += r.status == SolverStatus.SOLVED
        dt = time.perf_counter() - t0
        plain = {"value": nsol / dt, "unit": "solves/s", "sample": args.plain_sample,
                 "p50_ms": 1000 * float(np.percentile(lat, 50)),
                 "p99_ms": 1000 * float(np.percentile(lat, 99)), "method": "cudss",
                 "note": "per-solve latency back to back, no queue"}
        plain_lat = lat

    # ---- served: continuous batching under a Poisson request stream
    served = None
    if rank == 0 and args.serve_seconds > 0:
        try:
            served = serve_config5(pbs, args.serve_rate, args.serve_seconds, 12345 + rank,
                                   args.method, args.serve_budget_gb, args.serve_new_frac,
                                   args.serve_large_frac, args.serve_grace, args.plain_pool)
            if plain:
                served["vs_plain_solves"] = served["value"] / plain["value"]
        except Exception as ex:  # reported in the line; the other sections stand
            served = {"error": "%s: %s" % (type(ex).__name__, ex)}
            print("serving run failed: %r" % ex, file=sys.stderr, flush=True)

    # ---- roofline: the dominant device phase (an LDL kernel), plus the
    # update_scaling cone kernels for reference
    peaks, peak_kind = load_peaks()
    hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    peak_note = ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                 else "fallback 6.65 TB/s")
    phases = prof["phases"]
    dom = max(phases.items(), key=lambda kv: kv[1][0])
    kernels = {"ldl_solve": "k_ldl_solve_warp<double, 1> (single-warp LDL solve + refinement)",
               "ldl_solve2": "k_ldl_solve_warp<double, 2> (single-warp LDL solve of the "
                             "constant and affine right-hand sides + refinement)",
               "ldl_factor": "k_ldl_factor_stream (streamed LDL factorisation, 4 warps per "
                             "instance)"}
    summaries = {"ldl_solve": "ldl_solve_mpc4096.md", "ldl_solve2": "ldl_solve2_mpc4096.md",
                 "ldl_factor": "ldl_factor_stream_mpc4096.md"}

    def roofline(name):
        ms, calls = phases[name]
        by = prof["bytes"].get(name, 0.0)
        ach = by / (ms / 1000.0) / 1e9 if ms > 0 else 0.0
        return {"bound": "hbm", "kernel": kernels.get(name, name), "achieved": ach,
                "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": ncu_traffic(summaries[name]) if name in summaries else None,
                "traffic_source": ("profiles/" + summaries[name] + " (one captured launch; "
                                   "dram__bytes_read.sum + dram__bytes_write.sum)")
                if name in summaries else None,
                "peak_kind": peak_note,
                "algorithmic_bytes_per_launch": by / max(calls, 1),
                "avg_launch_ms": ms / max(calls, 1), "launches": calls}
    us_ms, us_calls = phases["update_scaling"]
    us_bytes = algorithmic_bytes_update_scaling(pbs)
    us_ach = us_bytes / (us_ms / max(us_calls, 1) / 1000.0) / 1e9 if us_ms > 0 else 0.0

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, (ref_solved, ref_obj) = cpu_baseline_sample(args.ref_sample)
        for meth, r32 in mixed_res.items():
            mixed[meth]["obj_rel_err_vs_oracle"] = obj_errors(r32, ref_solved, ref_obj)

    large = None
    if rank == 0 and args.large_scale > 0:
        pk = fp64_gemm_peak()
        large = {"fp64_gemm_tflops": pk}
        for which in (2, 3):
            try:
                large["config%d" % which] = large_single(
                    which, args.large_scale, args.method, sh, pk,
                    0 if args.no_cpu else args.large_cpu_scale)
            except Exception as ex:  # reported in the line; the other sections stand
                large["config%d" % which] = {"error": "%s: %s" % (type(ex).__name__, ex)}
                print("config %d run failed: %r" % (which, ex), file=sys.stderr, flush=True)

    cones = None
    if rank == 0 and args.cone_scale > 0:
        ck = cone_kernel_roofline(hbm, args.cone_scale, args.cone_reps)
        fr = sorted(v["frac"] for t in ck.values() for v in t["ops"].values())
        cones = {"workload": "one cone-level handle per type (plain path, B = 1): "
                             + ", ".join("%s %d cones x dim %d" % (k, v["cones"], v["dim"])
                                         for k, v in ck.items()),
                 "peak_gbs": hbm, "peak_kind": peak_note,
                 "timing": "CUDA events around each operation's kernels, median of %d, "
                           "L2 flushed before each call" % args.cone_reps,
                 "frac_median": fr[len(fr) // 2], "types": ck}

    if rank == 0:
        roof_name = dom[0] if dom[0] in kernels else "ldl_solve"
        roof = roofline(roof_name)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"cudssmixed": "f64 (LDL factorisation f32)",
                      "mixed_f64elim": "f64 (LDL factor stored f32)"}.get(args.method, "f64"),
            "data": "synthetic (seeded PCG64, MPC batch shapes)",
            "config": dict(workload_config(B, args.method),
                           l2="flushed (256 MB write) between timed steps",
                           device_bytes=dev_bytes, launch_shapes=launch_shapes),
            "e2e": {"value": e2e_val, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": "update_data! of every value (P, q, A, b) from pinned host "
                            "memory + solve! + all solutions (copied to pinned host staging, "
                            "read through views) and infos to the host, per step; solvers "
                            "set up beforehand, as on the reference arm"},
            "e2e_cold": cold,
            "gpu_launches": launches_per_solve * args.steps,
            "roofline": roof,
            "roofline_other": dict(
                {nm: roofline(nm) for nm in kernels
                 if nm != roof_name and phases.get(nm, (0.0, 0))[1] > 0},
                update_scaling={"achieved": us_ach, "frac": us_ach / hbm, "unit": "GB/s",
                                "algorithmic_bytes_per_launch": us_bytes,
                                "avg_launch_ms": us_ms / max(us_calls, 1)}),
            "phases_ms": {k: round(v[0], 3) for k, v in phases.items()},
            "dominant_phase": {"name": dom[0], "ms": dom[1][0], "calls": dom[1][1]},
            "batch": {"status": status_counts, "iters_mean": float(np.mean(iters)),
                      "iters_max": int(np.max(iters)),
                      "batch_latency_ms": 1000 * elapsed / args.steps},
            "mixed_precision": mixed,
            "plain_gpu": plain,
            "batched_vs_plain": (value / plain["value"]) if plain else None,
            "served": served,
            "cpu_baseline": cpu,
            "cone_kernels": cones,
            "large_single": large,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
