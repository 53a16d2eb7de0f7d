"""Sharding of independent simulations over ranks, run as a world-size-2
gloo job on CPU: the assignment is identical on every rank, disjoint,
complete and balanced, and the timing reduction takes the max over ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from hormone_b200 import shard  # noqa: E402


def test_assign_is_a_balanced_partition():
    import numpy as np

    rng = np.random.default_rng(3)
    w = (128 * 4 ** rng.uniform(size=512)) ** 2  # KH batch box sizes
    for world in (1, 2, 4, 8):
        parts = shard.assign(w, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        assert shard.imbalance(w, world) < 1.01
    assert shard.assign([5, 1, 1, 1], 2) == [[0], [1, 2, 3]]
    assert shard.assign([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.assign([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, weights, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard.my_share(weights, rank, world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        t = shard.max_over_ranks(10.0 + rank, dist)
        n = shard.sum_over_ranks(len(mine), dist)
        q.put((rank, got, t, n))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharding():
    world = 2
    weights = [float(x) for x in (300, 20, 20, 5, 120, 64, 64, 7, 1, 90)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, weights, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts = res[0][1]
    assert res[1][1] == parts  # every rank computed the same assignment
    assert sorted(parts[0] + parts[1]) == list(range(len(weights)))
    assert not set(parts[0]) & set(parts[1])
    for rank, _, t, n in res:
        assert t == 11.0  # max over ranks
        assert n == len(weights)
