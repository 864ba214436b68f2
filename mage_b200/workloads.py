"""Benchmark workloads of the GAMERA step (synthetic inputs of the stated shapes)."""
from __future__ import annotations

from mage_b200 import grids
from mage_b200.gamera import GameraGPU, GamParams, FP64

WORKLOADS = {
    "blast192": {"N": (192, 192, 192), "problem": "bw",
                 "desc": "3-D MHD blast wave, curvilinear periodic 192^3 (200^3 with ghosts), configs[1]"},
    "blast96": {"N": (96, 96, 96), "problem": "bw",
                "desc": "3-D MHD blast wave, curvilinear periodic 96^3 (profiling size)"},
    "ot128": {"N": (128, 128, 4), "problem": "ot", "desc": "Orszag-Tang 128x128x4, periodic, configs[0]"},
}


def corners(w):
    N = w["N"]
    return grids.warped_periodic_corners(*N) if w["problem"] == "bw" else grids.uniform_corners(*N)


def make_app(name: str, precision: int = FP64, strict: bool = False, xyz=None) -> GameraGPU:
    """GPU app with the workload's grid and initial condition (all set up on the device)."""
    w = WORKLOADS[name]
    N = w["N"]
    g = GameraGPU(GamParams(*N, do25D=(N[2] == 1), precision=precision, strict=strict))
    g.set_geometry(corners(w) if xyz is None else xyz)
    if w["problem"] == "bw":
        g.init_blast_wave()
    else:
        g.init_orszag_tang()
    return g
