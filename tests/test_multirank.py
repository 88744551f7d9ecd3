"""bench.py's multi-rank plumbing on CPU: two gloo ranks, barrier and the
max-over-ranks reduction used for timing (one process per GPU on a box)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, results):
    import datetime
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    assert bench.dist_env() == (rank, world, rank)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        t = bench.reduce_max(1.5 + rank, world, "cpu")
        results[rank] = t
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_rank_max_reduction():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    results = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(results) == {0: 2.5, 1: 2.5}


def test_single_rank_is_identity():
    import bench
    assert bench.reduce_max(3.0, 1) == 3.0
    bench.barrier(1)
