"""The multi-rank host logic of bench.py on CPU: two gloo ranks (no GPU).

Under torchrun every rank builds and queries its own copy of the scene (independent objects, no collective on
the data path); the only collectives are the barrier around the timed region and the max over ranks of the
device time. The reference arm runs on rank 0 only; the other ranks return without work.
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        m = bench.max_over_ranks(1.5 + rank, world)
        # a rank other than 0 does no work in the reference arm
        args = type("A", (), {"steps": 1, "warmup": 0})()
        ref = bench.run_reference(args, world, rank) if rank != 0 else "skipped"
        bench.barrier(world)
        q.put((rank, m, ref))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_barrier():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [2.5, 2.5]  # every rank sees the slowest rank's time
    assert got[1][2] is None
