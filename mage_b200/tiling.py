"""Multi-GPU tiling of the GAMERA step: the grid is cut into tiles along i, j
and k, one tile per GPU (one process per GPU), with the depth-4 halo exchange
and the dt reduction of the reference's MPI step (gamAppMpi_T,
src/gamera/gamapp_mpi.F90: 495-512 dt AllReduce(MIN), 573-782 updateMpiBCs /
haloUpdate). ``Slabs`` is the decomposition along k alone.

A tile has GAM_BC_HALO on every side that faces a neighbour (both sides of a
periodic direction that is cut) and the grid's own boundary kinds on the
others. A step on every tile, all of it enqueued on one CUDA stream with no
host synchronisation until the status check at the end of the steps:
``gam_step_begin_dev`` (predictor .. cell update), the tile's dt candidate
into a device tensor, the reduction over tiles (MIN of the IEEE bits of a
positive double, SUM of the bad-cell count; an NCCL all-reduce in place across
ranks), ``gam_step_end_dev`` reading the reduced values (dt decision, the
tile's own boundaries; every tile takes the same decision), then the halo
exchange direction by direction, I, then J, then K: pack the 4 layers next to
each halo side into a device buffer, send/receive with the neighbours (NCCL
point-to-point through torch.distributed, ordered after the pack on the same
stream), unpack into the ghost layers and recompute their Bxyz. A pack spans
the whole ghosted extent of the other two directions, so the later directions
carry the edge and corner ghosts the earlier ones filled. A failed step halts
the later kernels on the device and is reported by ``gam_step_status`` on
every tile.

``Tiles(..., comm=None)`` keeps all tiles in this process on one device and
swaps halos by device copies; it emulates the exchange for tests on one GPU
(no kernel waits for another). ``comm="dist"`` uses the default
torch.distributed process group, one tile per rank (rank = ti + pi (tj + pj
tk)). ``make_app`` replaces the GPU handle by another object with the same
methods (the CPU tests drive the orchestration over gloo with a host
stand-in).
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass

import numpy as np
import torch

from mage_b200.gamera import BC_HALO, BC_LFM, BC_PERIODIC, LIB_PATH, GameraGPU, GamParams

NG = 4


def tile_cut(a: np.ndarray, axis: int, n_active: int, parts: int, t: int) -> np.ndarray:
    """The part of array a that tile t of ``parts`` along one direction holds:
    a's extent along ``axis`` is n_active + e (e = 8 ghosts, 9 for corners or
    faces), the tile's n_active / parts + e starting at t n_active / parts."""
    n = n_active // parts
    e = a.shape[axis] - n_active
    sl = [slice(None)] * a.ndim
    sl[axis] = slice(t * n, t * n + n + e)
    return a[tuple(sl)]


def tile_box(a: np.ndarray, N, dims, t) -> np.ndarray:
    """The tile's block of a box array in C order (..., k, j, i) with ghosts
    (cells, faces or corners)."""
    for d, axis in ((0, -1), (1, -2), (2, -3)):
        a = tile_cut(a, a.ndim + axis, N[d], dims[d], t[d])
    return np.ascontiguousarray(a)


def tile_corners(xyz: np.ndarray, N, dims, t) -> np.ndarray:
    """Corners of tile t (Fortran layout (3, Nk+1, Nj+1, Ni+1) with ghosts)
    cut from the global corner array: its active cells plus 4 ghost layers on
    every side."""
    return tile_box(xyz, N, dims, t)


def slab_corners(xyz: np.ndarray, nslab: int, r: int) -> np.ndarray:
    """Corners of k-slab r: its nk active layers plus 4 ghost layers each side."""
    nk = (xyz.shape[1] - 1 - 2 * NG) // nslab
    return np.ascontiguousarray(xyz[:, r * nk:r * nk + nk + 2 * NG + 1])


@dataclass(frozen=True)
class Tile:
    """Tile index t = (ti, tj, tk) in a grid of dims tiles; n its active
    size; bc its six boundary kinds; edge per side whether it is an edge of
    the whole grid."""
    rank: int
    t: tuple
    n: tuple
    bc: tuple
    edge: tuple


class Tiles:
    """The tiles of one grid: all of them (comm=None) or this rank's (comm="dist").

    N the global active size, dims the tiles per direction (each must divide
    N), bc the grid's boundary kinds. problem: "bw" (the blast wave of
    gam_init_blast_wave on each tile, then the first exchange with Bxyz copied
    and the global dt), or a callable problem(g, tile) that completes the
    set-up of a handle whose geometry is set (fields, background, wind) and
    uploads its whole state with ghosts and its scalars (gam_upload_state).
    halo_dirs: the directions exchanged (default: those cut in more than one
    tile); a periodic direction in it with one tile sends to itself. rings:
    the keyword arguments of GameraGPU.set_rings for the tiles that hold an
    LFM pole (set before their geometry)."""

    def __init__(self, N, xyz: np.ndarray, dims, comm=None, precision: int = 0, strict: bool = False,
                 problem="bw", bc=None, lib_path: str = LIB_PATH, make_app=None, device=None, halo_dirs=None,
                 params: dict | None = None, rings: dict | None = None):
        self.N, self.dims = tuple(N), tuple(dims)
        for d in range(3):
            assert self.N[d] % self.dims[d] == 0, "the tiles must divide the grid"
        self.n = tuple(self.N[d] // self.dims[d] for d in range(3))
        self.ntile = int(np.prod(self.dims))
        self.gbc = tuple(bc) if bc is not None else (BC_PERIODIC,) * 6
        self.halo_dirs = tuple(halo_dirs) if halo_dirs is not None else tuple(d for d in range(3) if self.dims[d] > 1)
        for d in range(3):
            if self.dims[d] > 1 and d not in self.halo_dirs:
                raise ValueError("a direction cut into tiles exchanges halos")
            if d in self.halo_dirs and self.dims[d] == 1 and self.gbc[2 * d] != BC_PERIODIC:
                raise ValueError("one tile exchanges with itself only in a periodic direction")
        self.comm = comm
        if comm is None:
            self.ranks = list(range(self.ntile))
        else:
            import torch.distributed as dist
            self.dist = dist
            self.ranks = [dist.get_rank()]
            assert dist.get_world_size() == self.ntile
        self.tiles = [self.tile(r) for r in self.ranks]
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        # one stream for every tile's kernels, the reductions and the exchange
        self.stream = torch.cuda.Stream(self.device) if self.device.type == "cuda" else None

        def make_gpu_app(r):
            tl = self.tile(r)
            g = GameraGPU(GamParams(*self.n, bc=tl.bc, precision=precision, strict=strict, **(params or {})),
                          lib_path=lib_path)
            g.set_stream(self.stream.cuda_stream)
            for d in range(3):
                if tl.bc[2 * d] == BC_HALO or tl.bc[2 * d + 1] == BC_HALO:
                    g.set_tile_edges(d, tl.edge[2 * d], tl.edge[2 * d + 1])
            if BC_LFM in tl.bc[2:4]:
                g.set_rings(**(rings or {}))
            g.set_geometry(tile_corners(xyz, self.N, self.dims, tl.t))
            if problem == "bw":
                g.init_blast_wave()
            elif callable(problem):
                problem(g, tl)
            else:
                raise ValueError(problem)
            return g

        make = make_app if make_app is not None else make_gpu_app
        with self._on_stream():
            self.apps = [make(r) for r in self.ranks]
            self.buf = []
            for tl, g in zip(self.tiles, self.apps):
                bd = {}
                for d in self.halo_dirs:
                    nb = g.tile_halo_bytes(d)
                    bd[d] = {k: torch.empty(nb, dtype=torch.uint8, device=self.device)
                             for k in ("send0", "send1", "recv0", "recv1")}
                self.buf.append(bd)
            # per tile: dt candidate bits and bad-cell count
            self.part = torch.zeros((len(self.apps), 2), dtype=torch.int64, device=self.device)
            if problem == "bw" or make_app is not None:
                self.exchange(copyB=True)
                dts = [g.init_finish_halo() for g in self.apps]
                dt = self._allreduce_min_f(min(dts))
                for g in self.apps:
                    g.set_start(dt)

    # --- geometry of the decomposition ----------------------------------------------
    def index(self, r: int) -> tuple:
        pi, pj, _ = self.dims
        return (r % pi, (r // pi) % pj, r // (pi * pj))

    def rank_of(self, t) -> int:
        pi, pj, _ = self.dims
        return t[0] + pi * (t[1] + pj * t[2])

    def tile(self, r: int) -> Tile:
        t = self.index(r)
        bc, edge = [], []
        for d in range(3):
            per = self.gbc[2 * d] == BC_PERIODIC
            lo_edge, hi_edge = t[d] == 0, t[d] == self.dims[d] - 1
            ex = d in self.halo_dirs
            bc.append(BC_HALO if ex and (per or not lo_edge) else self.gbc[2 * d])
            bc.append(BC_HALO if ex and (per or not hi_edge) else self.gbc[2 * d + 1])
            edge += [lo_edge, hi_edge]
        return Tile(r, t, self.n, tuple(bc), tuple(edge))

    def neighbour(self, t, d: int, step: int):
        """Rank of the tile next to t in direction d (step -1 below, +1 above),
        wrapping a periodic direction; None past the grid's edge."""
        u = list(t)
        u[d] += step
        if not 0 <= u[d] < self.dims[d]:
            if self.gbc[2 * d] != BC_PERIODIC:
                return None
            u[d] %= self.dims[d]
        return self.rank_of(u)

    def _on_stream(self):
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    # --- reductions -------------------------------------------------------------
    def _allreduce_min_f(self, x: float) -> float:
        if self.comm is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        return float(t.item())

    def _reduce_dt(self):
        """Min of the candidates' bits and sum of the bad-cell counts over the
        tiles, as device tensors (gamapp_mpi.F90:495-512)."""
        bits = torch.amin(self.part[:, 0], dim=0, keepdim=True)
        nbad = torch.sum(self.part[:, 1], dim=0, keepdim=True)
        if self.comm is not None and self.ntile > 1:
            self.dist.all_reduce(bits, op=self.dist.ReduceOp.MIN)
            self.dist.all_reduce(nbad, op=self.dist.ReduceOp.SUM)
        return bits, nbad

    # --- halo exchange ----------------------------------------------------------
    def _sides(self, tl: Tile, d: int):
        return [s for s in (0, 1) if tl.bc[2 * d + s] == BC_HALO]

    def exchange(self, copyB: bool = False):
        """Halo exchange of every tile, direction by direction (I, J, K)."""
        with self._on_stream():
            for d in self.halo_dirs:
                for tl, g, b in zip(self.tiles, self.apps, self.buf):
                    for s in self._sides(tl, d):
                        g.tile_halo_pack(d, s, b[d]["send%d" % s])
                if self.comm is None or self.ntile == 1:
                    where = {tl.rank: q for q, tl in enumerate(self.tiles)}
                    for tl, b in zip(self.tiles, self.buf):
                        if tl.bc[2 * d] == BC_HALO:
                            b[d]["recv0"].copy_(self.buf[where[self.neighbour(tl.t, d, -1)]][d]["send1"])
                        if tl.bc[2 * d + 1] == BC_HALO:
                            b[d]["recv1"].copy_(self.buf[where[self.neighbour(tl.t, d, +1)]][d]["send0"])
                else:
                    tl = self.tiles[0]
                    up = self.neighbour(tl.t, d, +1) if tl.bc[2 * d + 1] == BC_HALO else None
                    down = self.neighbour(tl.t, d, -1) if tl.bc[2 * d] == BC_HALO else None
                    exchange_pair(self.dist, up, down, self.buf[0][d])
                for tl, g, b in zip(self.tiles, self.apps, self.buf):
                    for s in self._sides(tl, d):
                        g.tile_halo_unpack(d, s, b[d]["recv%d" % s], copyB)

    # --- stepping ---------------------------------------------------------------
    def step(self, n: int = 1):
        """n steps of every tile; returns (Model%dt, Model%t). Raises the
        GamError of a failed step, which every tile reports alike."""
        with self._on_stream():
            for _ in range(n):
                for g in self.apps:
                    g.step_begin_dev()
                for r, g in enumerate(self.apps):
                    g.dt_partial_dev(self.part[r, 0:1], self.part[r, 1:2])
                bits, nbad = self._reduce_dt()
                for g in self.apps:
                    g.step_end_dev(bits, nbad)
                self.exchange()
        return self.status()

    def status(self):
        out, err = [], None
        for g in self.apps:
            try:
                out.append(g.step_status())
            except Exception as e:  # every tile took the same decision; check them all
                err = e
        if err is not None:
            raise err
        return out[0]

    def last_step_ms(self) -> float:
        return max(g.last_step_ms() for g in self.apps)


class Slabs(Tiles):
    """The grid cut along k alone into nslab slabs (periodic in k; with one
    slab the halo goes to itself)."""

    def __init__(self, N, xyz: np.ndarray, nslab: int, comm=None, precision: int = 0, strict: bool = False,
                 problem: str = "bw", lib_path: str = LIB_PATH, make_app=None, device=None):
        self.nslab = nslab
        self.nk = N[2] // nslab
        super().__init__(N, xyz, (1, 1, nslab), comm=comm, precision=precision, strict=strict, problem=problem,
                         lib_path=lib_path, make_app=make_app, device=device, halo_dirs=(2,))


def exchange_pair(dist, up, down, b: dict):
    """Point-to-point halo swap with the tiles above (rank ``up``) and below
    (``down``) in one direction; None where the side is the grid's edge. Per
    rank the operations are: send up, receive from below, send down, receive
    from above; with two tiles in a periodic direction both neighbours are the
    same rank and the messages pair in this order."""
    ops = []
    if up is not None:
        ops.append(dist.P2POp(dist.isend, b["send1"], up))
    if down is not None:
        ops.append(dist.P2POp(dist.irecv, b["recv0"], down))
        ops.append(dist.P2POp(dist.isend, b["send0"], down))
    if up is not None:
        ops.append(dist.P2POp(dist.irecv, b["recv1"], up))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def exchange_dist(dist, rank: int, n: int, b: dict):
    """The k-slab swap: neighbours (rank +- 1) mod n, periodic in k."""
    exchange_pair(dist, (rank + 1) % n, (rank - 1) % n, b)
