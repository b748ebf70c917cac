"""The multi-rank plumbing of bench.py on CPU (gloo, two ranks): the path runs
one independent replica per GPU ("replicas only": no data-path collective), so
what the ranks share is the barrier around the timed region, the maximum of
the per-rank times and the record rank 0 prints.  The reference arm runs on
rank 0 alone."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier()
        t_max = bench.dist_max(0.25 + 0.5 * rank)     # per-rank "ms per step"
        bench.barrier()
        w = dict(bench.WORKLOADS["standard"])
        cfg = bench.bench_config(w, world, 4, 0)
        q.put((rank, t_max, cfg["parallelism"], cfg["global_batch"]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_the_max_time_and_the_replica_record():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[0] for g in got] == [0, 1]
    # every rank times the job with the slowest rank's time
    assert all(g[1] == 0.75 for g in got)
    assert all(g[2] == "replicas x2" and g[3] == 2 for g in got)


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")

    class Args:
        steps, warmup = 3, 3

    bench.run_reference(Args, dict(bench.WORKLOADS["standard"]))
    assert capsys.readouterr().out == ""
