"""Multi-GPU tiling of the GAMERA step: the grid is cut into slabs along k, one
slab per GPU (one process per GPU), with the depth-4 halo exchange and the dt
reduction of the reference's MPI step (gamAppMpi_T, src/gamera/gamapp_mpi.F90:
495-512 dt AllReduce(MIN), 573-782 updateMpiBCs / haloUpdate) for a
decomposition along k with periodic k.

A step on every slab, all of it enqueued on one CUDA stream with no host
synchronisation until the status check at the end of the steps:
``gam_step_begin_dev`` (predictor .. cell update), the slab's dt candidate
into a device tensor, the reduction over slabs (MIN of the IEEE bits of a
positive double, SUM of the bad-cell count; an NCCL all-reduce in place across
ranks), ``gam_step_end_dev`` reading the reduced values (dt decision, local
boundaries; every slab takes the same decision), then the halo exchange: pack
the 4 layers next to each k side into a device buffer, send/receive with the
neighbours (NCCL point-to-point through torch.distributed, ordered after the
pack on the same stream), unpack into the ghost layers and recompute their
Bxyz. A failed step halts the later kernels on the device and is reported by
``gam_step_status`` on every slab.

``Slabs(..., comm=None)`` keeps all slabs in this process on one device and
swaps halos by device copies; it emulates the exchange for tests on one GPU
(no kernel waits for another). ``comm="dist"`` uses the default
torch.distributed process group, one slab per rank. ``make_app`` replaces the
GPU handle by another object with the same methods (the CPU tests drive the
orchestration over gloo with a host stand-in).
"""
from __future__ import annotations

import contextlib

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
                 problem: str = "bw", lib_path: str = LIB_PATH, make_app=None, device=None):
        Nip, Njp, Nkp = N
        assert Nkp % nslab == 0, "Nkp must divide into the slabs"
        self.nslab, self.comm = nslab, comm
        self.nk = Nkp // nslab
        if comm is None:
            self.ranks = list(range(nslab))
        else:
            import torch.distributed as dist
            self.dist = dist
            self.ranks = [dist.get_rank()]
            assert dist.get_world_size() == nslab
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        # one stream for every slab's kernels, the reductions and the exchange
        self.stream = torch.cuda.Stream(self.device) if self.device.type == "cuda" else None

        def make_gpu_app(r):
            bc = (BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_HALO, BC_HALO)
            g = GameraGPU(GamParams(Nip, Njp, self.nk, bc=bc, precision=precision, strict=strict), lib_path=lib_path)
            g.set_stream(self.stream.cuda_stream)
            g.set_slab_edges(r == 0, r == nslab - 1)
            g.set_geometry(slab_corners(xyz, nslab, r))
            if problem == "bw":
                g.init_blast_wave()
            else:
                raise ValueError(problem)
            return g

        make = make_app if make_app is not None else make_gpu_app
        with self._on_stream():
            self.apps = [make(r) for r in self.ranks]
            nb = self.apps[0].halo_bytes()
            self.buf = [{k: torch.empty(nb, dtype=torch.uint8, device=self.device)
                         for k in ("send0", "send1", "recv0", "recv1")} for _ in self.apps]
            # per slab: dt candidate bits and bad-cell count
            self.part = torch.zeros((len(self.apps), 2), dtype=torch.int64, device=self.device)
            self.exchange(copyB=True)
            dts = [g.init_finish_halo() for g in self.apps]
            dt = self._allreduce_min_f(min(dts))
            for g in self.apps:
                g.set_start(dt)

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
        slabs, as device tensors (gamapp_mpi.F90:495-512)."""
        bits = torch.amin(self.part[:, 0], dim=0, keepdim=True)
        nbad = torch.sum(self.part[:, 1], dim=0, keepdim=True)
        if self.comm is not None and self.nslab > 1:
            self.dist.all_reduce(bits, op=self.dist.ReduceOp.MIN)
            self.dist.all_reduce(nbad, op=self.dist.ReduceOp.SUM)
        return bits, nbad

    # --- halo exchange ----------------------------------------------------------
    def exchange(self, copyB: bool = False):
        with self._on_stream():
            for g, b in zip(self.apps, self.buf):
                g.halo_pack(0, b["send0"])
                g.halo_pack(1, b["send1"])
            if self.comm is None or self.nslab == 1:
                n = len(self.apps)
                for r in range(n):
                    self.buf[r]["recv0"].copy_(self.buf[(r - 1) % n]["send1"])
                    self.buf[r]["recv1"].copy_(self.buf[(r + 1) % n]["send0"])
            else:
                exchange_dist(self.dist, self.ranks[0], self.nslab, self.buf[0])
            for g, b in zip(self.apps, self.buf):
                g.halo_unpack(0, b["recv0"], copyB)
                g.halo_unpack(1, b["recv1"], copyB)

    # --- stepping ---------------------------------------------------------------
    def step(self, n: int = 1):
        """n steps of every slab; returns (Model%dt, Model%t). Raises the
        GamError of a failed step, which every slab reports alike."""
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
            except Exception as e:  # every slab took the same decision; check them all
                err = e
        if err is not None:
            raise err
        return out[0]

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
