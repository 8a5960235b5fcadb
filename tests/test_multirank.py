"""The multi-GPU bench path on CPU ranks (gloo, world size 2): instance
shards do not overlap, and the whole-job figures are the slowest rank's time
and the sum of every rank's solves."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    t, s = bench.aggregate_over_ranks(1.5 + rank, 7 * (rank + 1), dist, "cpu")
    out.put((rank, t, s, bench.rank_seed0(rank, 4096)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_cpu_ranks_aggregate_and_shard():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    for _, t, s, _ in res:
        assert t == 2.5 and s == 21          # max over ranks, sum over ranks
    assert [r[3] for r in res] == [0, 4096]  # disjoint instance ranges


def _solve_worker(rank, world, port, per_rank, out):
    """One rank of the weak-scaling data plane: it takes its shard of the
    workload (instances rank_seed0 .. + per_rank), solves each one (here with
    the CPU oracle, standing in for the rank's GPU), and joins the whole-job
    figures (max time, summed solves) with no other collective."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import time
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    import oracle
    from cuclarabel_b200 import problems
    seed0 = bench.rank_seed0(rank, per_rank)
    t0 = time.perf_counter()
    ids, solved = [], 0
    for pb, i in zip(problems.mpc_batch(per_rank, seed0=seed0), range(seed0, seed0 + per_rank)):
        r = oracle.solve(*pb, gpu_equilibration=1)
        ids.append(i)
        solved += r["status_name"] == "SOLVED"
    t, s = bench.aggregate_over_ranks(time.perf_counter() - t0, solved, dist, "cpu")
    out.put((rank, ids, solved, s, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_cpu_ranks_solve_their_shards():
    import oracle
    from cuclarabel_b200 import problems
    per_rank = 3
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_solve_worker, args=(r, 2, port, per_rank, out))
             for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ids = [i for r in res for i in r[1]]
    assert len(ids) == len(set(ids)) == 2 * per_rank       # shards do not overlap
    total = sum(r[2] for r in res)
    assert all(r[3] == total for r in res)                  # every rank sees the job sum
    assert res[0][4] == res[1][4] > 0                       # and the slowest rank's time
    # the same instances solved in one process give the same count
    single = sum(oracle.solve(*problems.mpc_qp(i), gpu_equilibration=1)["status_name"] == "SOLVED"
                 for i in ids)
    assert total == single
