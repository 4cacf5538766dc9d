"""The multi-GPU path of bench.py on CPU: replicas only (every rank evaluates its own copy of the workload, no
collective on the data path), timed as the maximum over ranks, reported by rank 0 as whole-job throughput
(world x steps / max time).  Two gloo ranks on 127.0.0.1 check the pieces bench.py uses for that: the max-over-ranks
reduction, the barrier around the timed region, and that the reference arm does its work on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        t = bench.reduce_max(1.5 + rank, world)           # each rank's timed seconds; the job's time is the max
        bench.barrier(world)
        steps = 10
        value = world * steps / t                          # whole-job evaluations per second
        ran = bench.run_reference(type("A", (), {})(), world, rank) if rank else "skipped"
        q.put((rank, t, value, ran))
    finally:
        dist.destroy_process_group()


def test_replicas_max_over_ranks_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]               # both ranks see the slowest rank's time
    assert out[0][2] == pytest.approx(2 * 10 / 2.5)
    assert out[1][3] is None                               # rank 1: the reference arm returns without work
