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


def test_scene_partition_covers_every_scene_once():
    """The batched workload's scene-parallel sharding: every scene on exactly
    one rank, and the greedy largest-first assignment within one scene of the
    even share."""
    sys.path.insert(0, os.path.join(ROOT, "ar-physics_b200"))
    import numpy as np
    from arphys import scenes
    rng = np.random.default_rng(5)
    sizes = np.round(np.exp(rng.uniform(np.log(2048), np.log(65536), size=256))).astype(int)
    for world in range(1, 9):
        parts = scenes.partition_scenes(sizes, world)
        assert len(parts) == world
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        loads = [int(sizes[p].sum()) for p in parts]
        assert max(loads) <= sizes.sum() / world + sizes.max()
    with pytest.raises(ValueError):
        scenes.partition_scenes(sizes, 0)


def _partition_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "ar-physics_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    from arphys import scenes
    sizes = [sc.n + sc.nb for sc in scenes.batched_scenes(count=32, n_max=4096)]
    mine = scenes.partition_scenes(sizes, world)[rank]
    got = [None] * world
    torch.distributed.all_gather_object(got, mine)
    out[rank] = got
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()


def test_two_ranks_take_disjoint_shares_of_the_batch():
    """Each rank computes its share on its own (no exchange); the shares the
    ranks arrive at are disjoint and cover the batch."""
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_partition_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    assert out[0] == out[1]
    a, b = out[0]
    assert not set(a) & set(b) and sorted(a + b) == list(range(32))
