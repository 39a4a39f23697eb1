"""The multi-rank path of bench.py on CPU: two gloo ranks, each timing its own
replica, combine into one whole-job rate using the slowest rank's time."""
import os
import socket
import sys

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    import bench
    seconds = 2.0 + rank  # rank 1 is the slow one
    t = bench.max_over_ranks(seconds, "cpu")
    out[rank] = bench.aggregate_rate(1000.0, world, t)
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()


def test_two_rank_rate_uses_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == pytest.approx(1000.0 * 2 / 3.0)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(1.5, "cpu") == 1.5
