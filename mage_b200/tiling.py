"""Multi-GPU tiling of the GAMERA step: the grid is cut into slabs along k, one
slab per GPU (one process per GPU), with the depth-4 halo exchange and the dt
reduction of the reference's MPI step (gamAppMpi_T, src/gamera/gamapp_mpi.F90:
495-512 dt AllReduce(MIN), 573-782 updateMpiBCs / haloUpdate) for a
decomposition along k with periodic k.

A step on every slab: ``gam_step_begin`` (predictor .. cell update), the
all-reduce of the dt candidate (min of the IEEE bits of a positive double, sum
of the bad-cell count), ``gam_step_end`` (dt decision, local boundaries), then
the halo exchange: pack the 4 layers next to each k side into a device buffer,
send/receive with the neighbours (NCCL point-to-point through
torch.distributed), unpack into the ghost layers and recompute their Bxyz.

``Slabs(..., comm=None)`` keeps all slabs in this process on one device and
swaps halos by device copies; it emulates the exchange for tests on one GPU
(no kernel waits for another). ``comm="dist"`` uses the default
torch.distributed process group, one slab per rank.
"""
from __future__ import annotations

import numpy as np
import torch

from mage_b200.gamera import BC_HALO, BC_PERIODIC, FP32, LIB_PATH, GameraGPU, GamParams

NG = 4


def slab_corners(xyz: np.ndarray, nslab: int, r: int) -> np.ndarray:
    """Corners of slab r (Fortran layout (3, Nk+1, Nj+1, Ni+1)) cut from the
    global corner array: its nk active layers plus 4 ghost layers each side."""
    nk = (xyz.shape[1] - 1 - 2 * NG) // nslab
    return np.ascontiguousarray(xyz[:, r * nk:r * nk + nk + 2 * NG + 1])


class Slabs:
    """The slabs of one grid: all of them (comm=None) or this rank's (comm="dist")."""

    def __init__(self, N, xyz: np.ndarray, nslab: int, comm=None, precision: int = 0, strict: bool = False,
                 problem: str = "bw", lib_path: str = LIB_PATH):
        Nip, Njp, Nkp = N
        assert Nkp % nslab == 0, "Nkp must divide into the slabs"
        self.nslab, self.comm = nslab, comm
        self.nk = Nkp // nslab
        if comm is None:
            self.ranks = list(range(nslab))
            self.device = torch.device("cuda", torch.cuda.current_device())
        else:
            import torch.distributed as dist
            self.dist = dist
            self.ranks = [dist.get_rank()]
            assert dist.get_world_size() == nslab
            self.device = torch.device("cuda", torch.cuda.current_device())
        bc = (BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_HALO, BC_HALO)
        self.apps = []
        for r in self.ranks:
            g = GameraGPU(GamParams(Nip, Njp, self.nk, bc=bc, precision=precision, strict=strict), lib_path=lib_path)
            g.set_slab_edges(r == 0, r == nslab - 1)
            g.set_geometry(slab_corners(xyz, nslab, r))
            if problem == "bw":
                g.init_blast_wave()
            else:
                raise ValueError(problem)
            self.apps.append(g)
        nb = self.apps[0].halo_bytes()
        self.buf = [{k: torch.empty(nb, dtype=torch.uint8, device=self.device)
                     for k in ("send0", "send1", "recv0", "recv1")} for _ in self.apps]
        self.exchange(copyB=True)
        dts = [g.init_finish_halo() for g in self.apps]
        dt = self._allreduce_min_f(min(dts))
        for g in self.apps:
            g.set_start(dt)

    # --- reductions -------------------------------------------------------------
    def _allreduce_min_f(self, x: float) -> float:
        if self.comm is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        return float(t.item())

    def _allreduce_dt(self, parts):
        bits = min(p[0] for p in parts)
        nbad = sum(p[1] for p in parts)
        if self.comm is None:
            return bits, nbad
        t = torch.tensor([bits], dtype=torch.int64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        n = torch.tensor([nbad], dtype=torch.int64, device=self.device)
        self.dist.all_reduce(n, op=self.dist.ReduceOp.SUM)
        return int(t.item()), int(n.item())

    # --- halo exchange ----------------------------------------------------------
    def exchange(self, copyB: bool = False):
        for g, b in zip(self.apps, self.buf):
            g.halo_pack(0, b["send0"].data_ptr())
            g.halo_pack(1, b["send1"].data_ptr())
        if self.comm is None or self.nslab == 1:
            n = len(self.apps)
            for r in range(n):
                self.buf[r]["recv0"].copy_(self.buf[(r - 1) % n]["send1"])
                self.buf[r]["recv1"].copy_(self.buf[(r + 1) % n]["send0"])
        else:
            exchange_dist(self.dist, self.ranks[0], self.nslab, self.buf[0])
        torch.cuda.current_stream().synchronize()
        for g, b in zip(self.apps, self.buf):
            g.halo_unpack(0, b["recv0"].data_ptr(), copyB)
            g.halo_unpack(1, b["recv1"].data_ptr(), copyB)

    # --- stepping ---------------------------------------------------------------
    def step(self, n: int = 1):
        dt = t = None
        for _ in range(n):
            for g in self.apps:
                g.step_begin()
            bits, nbad = self._allreduce_dt([g.dt_partial() for g in self.apps])
            err = None
            for g in self.apps:
                try:
                    dt, t = g.step_end(bits, nbad)
                except Exception as e:  # every slab took the same decision; finish them all
                    err = e
            if err is not None:
                raise err
            self.exchange()
        return dt, t

    def last_step_ms(self) -> float:
        return max(g.last_step_ms() for g in self.apps)


def exchange_dist(dist, rank: int, n: int, b: dict):
    """Point-to-point halo swap with the slabs below and above (periodic in k).
    Per rank the operations are: send up, receive from below, send down,
    receive from above; with two slabs both neighbours are the same rank and
    the messages pair in this order."""
    up, down = (rank + 1) % n, (rank - 1) % n
    ops = [dist.P2POp(dist.isend, b["send1"], up), dist.P2POp(dist.irecv, b["recv0"], down),
           dist.P2POp(dist.isend, b["send0"], down), dist.P2POp(dist.irecv, b["recv1"], up)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
