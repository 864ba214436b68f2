"""Host logic of the k-slab halo exchange (mage_b200.tiling.exchange_dist) on
CPU ranks over gloo: every rank receives its lower ghosts from the slab below
(that slab's upward pack) and its upper ghosts from the slab above, periodic
in k, with 2 ranks (both neighbours the same rank) and with 3."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from mage_b200.tiling import exchange_dist, slab_corners


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, n, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=n)
    try:
        b = {"send0": torch.full((8,), 10.0 * rank + 0), "send1": torch.full((8,), 10.0 * rank + 1),
             "recv0": torch.zeros(8), "recv1": torch.zeros(8)}
        exchange_dist(dist, rank, n, b)
        q.put((rank, float(b["recv0"][0]), float(b["recv1"][0])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [2, 3])
def test_exchange_pairs_neighbours(n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, n, port, q)) for r in range(n)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(n):
        rank, lo, hi = q.get(timeout=120)
        got[rank] = (lo, hi)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(n):
        assert got[r] == (10.0 * ((r - 1) % n) + 1, 10.0 * ((r + 1) % n) + 0), (r, got[r])


def test_slab_corners_overlap():
    import numpy as np
    from mage_b200 import grids
    xyz = grids.warped_periodic_corners(16, 16, 16)
    parts = [slab_corners(xyz, 4, r) for r in range(4)]
    for r, p in enumerate(parts):
        assert p.shape == (3, 4 + 9, 25, 25)
        assert np.array_equal(p, xyz[:, 4 * r:4 * r + 13])
