"""Benchmark workloads of the GAMERA step (synthetic inputs of the stated shapes)."""
from __future__ import annotations

from mage_b200 import dipole, grids
import numpy as np

from mage_b200.gamera import (BC_ION, BC_LFM, BC_PERIODIC, BC_SPHIN, BC_WIND, BC_ZEROGRAD, FP64, GameraGPU,
                              GamParams)

# inner sphere, solar wind, zero-gradient at the polar axis, periodic in phi
DIPOLE_BCS = (BC_SPHIN, BC_WIND, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)
# the magnetosphere: ionospheric inner boundary, solar wind, LFM pole at both J sides
MAGSPHERE_BCS = (BC_ION, BC_WIND, BC_LFM, BC_LFM, BC_PERIODIC, BC_PERIODIC)
ION_DTCPL = 5.0 / 63.8  # the coupling time scale (5 s in code time)

WORKLOADS = {
    "blast192": {"N": (192, 192, 192), "problem": "bw",
                 "desc": "3-D MHD blast wave, curvilinear periodic 192^3 (200^3 with ghosts)"},
    "blast96": {"N": (96, 96, 96), "problem": "bw",
                "desc": "3-D MHD blast wave, curvilinear periodic 96^3 (profiling size)"},
    "ot128": {"N": (128, 128, 4), "problem": "ot", "desc": "Orszag-Tang 128x128x4, periodic"},
    "dipole96": {"N": (96, 96, 128), "problem": "dipole",
                 "desc": "dipole in a constant solar wind, spherical 96x96x128 (r 2-30), background field, "
                         "inner-sphere / wind / zero-gradient / periodic boundaries"},
    "dipole192": {"N": (192, 192, 256), "problem": "dipole",
                  "desc": "dipole in a constant solar wind, spherical 192x192x256 (r 2-30), background field"},
    "lfm96": {"N": (96, 96, 128), "problem": "magsphere",
              "desc": "magnetosphere on an LFM-style grid 96x96x128 (spherical about x, r 2-30, first corner row "
                      "0.01 rad off the axis): ionospheric inner boundary with its hooks (quiet coupling fields), "
                      "constant solar wind, LFM pole at both J sides with the reference's default rings for 128 "
                      "cells around the axis, background dipole"},
}


def ion_fields(N):
    """Quiet coupling fields of the ionospheric boundary (zero E)."""
    return np.zeros((3, N[2] + 8, N[1] + 8, 5)), np.zeros((3, N[2] + 9, N[1] + 9, 6))


def corners(w):
    N = w["N"]
    if w["problem"] == "bw":
        return grids.warped_periodic_corners(*N)
    if w["problem"] == "dipole":
        return grids.spherical_corners(*N)
    if w["problem"] == "magsphere":
        return grids.lfm_corners(*N, th0=0.01)
    return grids.uniform_corners(*N)


def make_app(name: str, precision: int = FP64, strict: bool = False, xyz=None) -> GameraGPU:
    """GPU app with the workload's grid and initial condition (all set up on the device)."""
    w = WORKLOADS[name]
    N = w["N"]
    if w["problem"] == "dipole":
        g = GameraGPU(GamParams(*N, precision=precision, strict=strict, doBackground=True, bc=DIPOLE_BCS))
        g.set_geometry(corners(w) if xyz is None else xyz)
        g.set_background_dipole(dipole.M0)
        g.init_dipole_wind(dipole.wind_code_units())
        return g
    if w["problem"] == "magsphere":
        g = GameraGPU(GamParams(*N, precision=precision, strict=strict, doBackground=True, bc=MAGSPHERE_BCS))
        g.set_rings()
        g.set_geometry(corners(w) if xyz is None else xyz)
        g.set_background_dipole(dipole.M0)
        E, Ee = ion_fields(N)
        g.set_ionosphere(E, Ee, dipole.M0, ION_DTCPL, True, 1)
        g.init_dipole_wind(dipole.wind_code_units())
        return g
    g = GameraGPU(GamParams(*N, do25D=(N[2] == 1), precision=precision, strict=strict))
    g.set_geometry(corners(w) if xyz is None else xyz)
    if w["problem"] == "bw":
        g.init_blast_wave()
    else:
        g.init_orszag_tang()
    return g
