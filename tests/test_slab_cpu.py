"""Host side of the slab decomposition along z (hormone_b200/slab.py), as
world-size-2 and -3 gloo jobs on CPU: the partition, the neighbours, the
face-to-face pairing of the halo messages (periodic and not) and the
min/max reduction of the CFL partials."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from hormone_b200 import slab  # noqa: E402


def test_partition_and_neighbours():
    assert slab.partition(16, 2) == [(0, 8), (8, 16)]
    assert slab.partition(13, 3) == [(0, 5), (5, 9), (9, 13)]
    with pytest.raises(ValueError):
        slab.partition(5, 3)  # a slab needs the stencil's two layers
    assert slab.neighbours(0, 3, False) == (None, 1)
    assert slab.neighbours(2, 3, False) == (1, None)
    assert slab.neighbours(0, 3, True) == (2, 1)
    assert slab.neighbours(1, 2, True) == (0, 0)
    assert slab.neighbours(0, 1, True) == (None, None)


def test_push_links_pair_faces():
    """Push exchange: a slab's bottom layers go to its low neighbour's "hi"
    buffers and its top layers to the high neighbour's "lo" buffers; every
    buffer that a slab reads has exactly one writer."""
    assert slab.push_links(1, True) == [{"lo": None, "hi": None}]
    assert slab.push_links(3, False) == [{"lo": None, "hi": (1, "lo")}, {"lo": (0, "hi"), "hi": (2, "lo")},
                                         {"lo": (1, "hi"), "hi": None}]
    assert slab.push_links(2, True) == [{"lo": (1, "hi"), "hi": (1, "lo")}, {"lo": (0, "hi"), "hi": (0, "lo")}]
    for world in (2, 3, 5):
        for periodic in (False, True):
            links = slab.push_links(world, periodic)
            writers = {}
            for r, lk in enumerate(links):
                for face in ("lo", "hi"):
                    if lk[face] is not None:
                        assert lk[face] not in writers
                        writers[lk[face]] = r
            for r in range(world):
                lo, hi = slab.neighbours(r, world, periodic)
                assert writers.get((r, "lo")) == lo and writers.get((r, "hi")) == hi


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, periodic, q):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ex = slab.TorchExchange(dist, rank, world, periodic)
        n = 6
        send_lo = torch.full((n,), 100.0 * rank + 1.0)   # this slab's lowest layers
        send_hi = torch.full((n,), 100.0 * rank + 2.0)   # this slab's highest layers
        recv_lo, recv_hi = torch.full((n,), -1.0), torch.full((n,), -1.0)
        ex.halos(send_lo, send_hi, recv_lo, recv_hi)
        tmin = torch.tensor([10.0 + rank], dtype=torch.float64)
        tmax = torch.tensor([10.0 + rank], dtype=torch.float64)
        ex.cfl(tmin, tmax)
        unit = ex.min_scalar(0.5 + 0.25 * ((rank + 1) % world))  # the gravity unit's minimum over slabs
        q.put((rank, float(recv_lo[0]), float(recv_hi[0]), float(tmin), float(tmax), ex.lo, ex.hi, unit))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True)])
def test_gloo_halo_exchange_pairs_faces(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rlo, rhi, tmin, tmax, lo, hi, unit in res:
        assert unit == 0.5
        # the low halo holds the lower neighbour's highest layers, the high
        # halo the upper neighbour's lowest layers; physical faces are untouched
        assert rlo == (100.0 * lo + 2.0 if lo is not None else -1.0)
        assert rhi == (100.0 * hi + 1.0 if hi is not None else -1.0)
        assert tmin == 10.0 and tmax == 10.0 + world - 1
