"""The multi-rank plumbing of bench.py on CPU: two gloo ranks.

BFS does not shard, so `bench.py --gpus N` runs N independent replicas and
the only cross-rank steps are a barrier and the max over ranks of the timed
seconds (the job's time is its slowest rank's).  Both run here with the gloo
backend on 127.0.0.1; on the GPU box they run over NCCL.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        bench.barrier(world)
        secs = 0.25 + rank  # rank 1 is the slow one
        t = bench.max_over_ranks(secs, world)
        # value = units of all ranks / the slowest rank's time (weak scaling)
        q.put((rank, t, world * 100 / t))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [r for r, _, _ in got] == [0, 1]
    assert all(t == pytest.approx(1.25) for _, t, _ in got)
    assert all(v == pytest.approx(160.0) for _, _, v in got)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(0.5, 1) == 0.5
    bench.barrier(1)
