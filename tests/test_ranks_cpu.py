"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the
replicas agree on the slowest rank's time and on the whole-job rate, and
the reference arm does its work on rank 0 only.  The samplers themselves
do not shard across GPUs (independent chains / replicas), so these
reductions are the only cross-rank steps."""
import datetime
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    try:
        t = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        q.put((rank, t, bench.aggregate_rate(1000, world, t)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    assert [g[1] for g in got] == [2.5, 2.5]
    assert all(g[2] == pytest.approx(2000 / 2.5) for g in got)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.aggregate_rate(10, 1, 2.0) == 5.0


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.run_reference(None, rank=1, world=2) is None
