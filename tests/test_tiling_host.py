"""Host logic of the tiling on CPU ranks over gloo:

* the halo exchange (mage_b200.tiling.exchange_dist): every rank receives its
  lower ghosts from the slab below (that slab's upward pack) and its upper
  ghosts from the slab above, periodic in k, with 2 ranks (both neighbours the
  same rank) and with 3;
* the orchestration of Slabs.step with a host stand-in for the GPU handle:
  every rank finishes each step with the MIN of the slabs' dt bits and the
  SUM of their bad-cell counts (the dt AllReduce of gamapp_mpi.F90:495-512),
  takes the same failure decision when one rank holds a bad cell, and runs
  the calls of a step in the same order (begin, candidate, end, pack down,
  pack up, unpack lower, unpack upper);
* tiles in two directions (2 x 2 tiles, I non-periodic with the grid's own
  boundaries outside, J periodic): each tile's boundary kinds and grid-edge
  flags, and that every halo side receives the pack of the right neighbour,
  direction by direction, over gloo and in one process.
* the tile slicing (tile_box / tile_cut) against explicit index ranges."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from mage_b200.gamera import BC_HALO, BC_PERIODIC, BC_SPHIN, BC_WIND, BC_ZEROGRAD
from mage_b200.tiling import Tiles, exchange_dist, slab_corners, tile_box, tile_cut


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


class _FakeSlab:
    """Stands in for GameraGPU inside Slabs: the slab's dt candidate in step n
    is dt0 (1 + n/10) (1 + rank/100); plant_bad = (rank, step) gives that rank
    one bad cell in that step. The halo buffers carry 40 rank + 10 dir + side."""

    def __init__(self, rank, plant_bad=None, shared=None):
        self.rank, self.plant_bad = rank, plant_bad
        self.n, self.log, self.recv = 0, [], {}
        self.shared = shared if shared is not None else []  # (rank, event) of every stand-in, in call order
        self.failed, self.dt, self.seen = False, None, []

    def tile_halo_bytes(self, d):
        return 16

    def tile_halo_pack(self, d, side, buf):
        buf.fill_(40 * self.rank + 10 * d + side)  # < 256: the buffers are bytes
        self.log.append(("pack", side) if d == 2 else ("pack", d, side))
        self.shared.append((self.rank, "pack", d))

    def tile_halo_unpack(self, d, side, buf, copyB=False):
        self.recv[side if d == 2 else (d, side)] = int(buf[0])
        self.log.append(("unpack", side) if d == 2 else ("unpack", d, side))
        self.shared.append((self.rank, "unpack", d))

    def init_finish_halo(self):
        return 0.5 + self.rank

    def set_start(self, dt):
        self.start = dt

    def step_begin_dev(self):
        self.n += 1
        self.log.append(("begin",))

    def dt_partial_dev(self, bits, nbad):
        import struct
        dt = 1e-3 * (1 + self.n / 10) * (1 + self.rank / 100)
        bits[0] = struct.unpack("<q", struct.pack("<d", dt))[0]
        nbad[0] = 1 if self.plant_bad == (self.rank, self.n) else 0
        self.log.append(("partial",))

    def step_end_dev(self, bits, nbad):
        import struct
        self.seen.append((int(bits[0]), int(nbad[0])))
        self.dt = struct.unpack("<d", struct.pack("<q", int(bits[0])))[0]
        if int(nbad[0]) > 0:
            self.failed = True
        self.log.append(("end",))

    def step_status(self):
        from mage_b200.gamera import GamError
        if self.failed:
            raise GamError(5, "CalcDT: timestep too small or not finite")
        return self.dt, float(self.n)


def _slab_worker(rank, n, port, plant, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=n)
    try:
        from mage_b200.tiling import Slabs
        sl = Slabs((16, 16, 4 * n), None, n, comm="dist", device=torch.device("cpu"),
                   make_app=lambda r: _FakeSlab(r, plant))
        app = sl.apps[0]
        app.log.clear()
        code = 0
        try:
            dt, _ = sl.step(3)
        except Exception as e:  # the stand-in's GamError
            dt, code = None, getattr(e, "code", -1)
        q.put((rank, app.start, dt, code, app.seen, app.recv, app.log))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("plant", [None, (1, 2)], ids=["ok", "bad-cell-on-rank1"])
def test_slab_step_orchestration(plant):
    import struct
    n = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_worker, args=(r, n, port, plant, q)) for r in range(n)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(n):
        r = q.get(timeout=180)
        got[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    step = [("begin",), ("partial",), ("end",), ("pack", 0), ("pack", 1), ("unpack", 0), ("unpack", 1)]
    for r in range(n):
        start, dt, code, seen, recv, log = got[r]
        assert start == 0.5  # min over the slabs of the start dt
        assert log == step * 3
        assert recv == {0: 40 * ((r - 1) % n) + 21, 1: 40 * ((r + 1) % n) + 20}
        for k, (bits, nbad) in enumerate(seen):  # the reduced candidate of step k+1: rank 0's
            want = 1e-3 * (1 + (k + 1) / 10)
            assert bits == struct.unpack("<q", struct.pack("<d", want))[0], (r, k)
            assert nbad == (1 if plant is not None and plant[1] == k + 1 else 0)
        if plant is None:
            assert code == 0 and dt == 1e-3 * 1.3
        else:
            assert code == 5 and dt is None  # the same decision on every rank
    assert got[0][3] == got[1][3]  # both ranks saw the same reduced values every step


# --- tiles in two directions ------------------------------------------------------
GBC = (BC_SPHIN, BC_WIND, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC)
DIMS = (2, 2, 1)


def _want_tile(r):
    ti, tj = r % 2, r // 2
    bc = (BC_SPHIN if ti == 0 else BC_HALO, BC_WIND if ti == 1 else BC_HALO, BC_HALO, BC_HALO,
          BC_PERIODIC, BC_PERIODIC)
    # I: tile ti+1 sends its side-0 pack down, tile ti-1 its side-1 pack up;
    # J periodic with 2 tiles: both neighbours are the other tj
    other_j = ti + 2 * (1 - tj)
    recv = {(1, 0): 40 * other_j + 11, (1, 1): 40 * other_j + 10}
    if ti == 0:
        recv[(0, 1)] = 40 * (r + 1) + 0
    else:
        recv[(0, 0)] = 40 * (r - 1) + 1
    return bc, recv


def _tiles(comm, device, shared=None):
    return Tiles((32, 16, 8), None, DIMS, comm=comm, bc=GBC, device=device,
                 make_app=lambda r: _FakeSlab(r, shared=shared))


def test_tiles_in_one_process():
    shared = []
    tl = _tiles(None, torch.device("cpu"), shared)
    assert tl.halo_dirs == (0, 1)
    for r, (t, g) in enumerate(zip(tl.tiles, tl.apps)):
        bc, recv = _want_tile(r)
        assert t.bc == bc and t.n == (16, 8, 8), (r, t)
        assert t.edge == (t.t[0] == 0, t.t[0] == 1, t.t[1] == 0, t.t[1] == 1, True, True)
        assert g.recv == recv, (r, g.recv)
    # the I packs and unpacks of every tile come before any J pack
    first_j = min(i for i, e in enumerate(shared) if e[1:] == ("pack", 1))
    assert first_j > max(i for i, e in enumerate(shared) if e[1:] == ("unpack", 0))
    assert len(shared) == 2 * (4 + 8)  # I: one side per tile, J: two


def _tile_worker(rank, n, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=n)
    try:
        tl = _tiles("dist", torch.device("cpu"))
        app = tl.apps[0]
        q.put((rank, tl.tiles[0].bc, dict(app.recv), list(app.log)))
    finally:
        dist.destroy_process_group()


def test_tiles_exchange_over_gloo():
    n = 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_tile_worker, args=(r, n, port, q)) for r in range(n)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(n):
        r, bc, recv, log = q.get(timeout=180)
        got[r] = (bc, recv, log)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(n):
        bc, recv = _want_tile(r)
        assert got[r][0] == bc and got[r][1] == recv, (r, got[r])
        log = got[r][2]
        assert log.index(("pack", 1, 0)) > max(i for i, e in enumerate(log) if e[:2] == ("unpack", 0))


def test_tile_slicing():
    import numpy as np
    N, dims = (16, 8, 12), (2, 2, 3)
    a = np.arange(3 * 21 * 17 * 25, dtype=np.float64).reshape(3, 21, 17, 25)  # corners
    for t in ((0, 0, 0), (1, 1, 2), (1, 0, 1)):
        b = tile_box(a, N, dims, t)
        assert b.shape == (3, 4 + 9, 4 + 9, 8 + 9)
        assert np.array_equal(b, a[:, 4 * t[2]:4 * t[2] + 13, 4 * t[1]:4 * t[1] + 13, 8 * t[0]:8 * t[0] + 17])
    e = np.zeros((3, 20, 16, 5))
    assert tile_cut(e, 2, 8, 2, 1).shape == (3, 20, 12, 5)
