"""Input decks in the reference's XML format for the GPU step.

A deck is the ``<Kaiju><Gamera>`` block of the reference's input file: one
element per section, keys as attributes (``<sim pdmb="0.75" .../>``), read by
``Set_Val(var, 'section/key', default)`` (src/base/io_xml_input.F90), keys and
sections compared without regard to case, logicals read as Fortran list input
(``T``, ``F``, ``.true.`` ...). This module maps the keys the step honours onto
``GamParams`` with the reference's defaults:

  initModel (src/gamera/init.F90:312-484)
    physics/doMHD F, physics/do25D F, sim/pdmb 0.75,
    sim/CFL min(0.5/(pdmb+0.5), 0.3), sim/Vd0 0.5, physics/gamma 5/3,
    physics/doHogs T with physics/cHogH = physics/cHogM = 0.25 (0 without),
    sim/doAB3 F, time/tFin 1, time/fixedTimestep -1 (off),
    timestep/limDT0 1e-3, physics/doBoris F with physics/Ca HUGE,
    sim/rmeth 8CENT | 7UP, sim/lfmlim T
  SetFloors (src/gamera/gamutils.F90:387-405)
    sim/dFloor, then floors/dFloor; sim/pFloor, then floors/pFloor; TINY
  genGridXML (src/gamera/init.F90:564-790), uniform Cartesian only
    idir/jdir/kdir N, min, max
  the set-ups of src/gamera/prob.F90 via sim/icType
    OT2D (:74-119); BW (:190-298) with prob/x0, y0, z0 (0), D0 (1), P0 (0.1),
    pRat (100), dRat (1), rC (0.1), B0 (1); ADV1D (:671-736, physics/gamma
    defaults to 1.4 for it); ADV2D (:739-797) and LOOP2D (:436-500) with
    prob/V0 (1), alpha (60); ALFVEN (:1027-1083) with prob/alp (pi/3); their
    other prob/ keys at the reference's defaults

Keys that switch on parts the GPU step does not have (resistivity,
multifluid, CPR, curvilinear grid generators, HDF5 grids or restarts, a moving
blast wave) raise ValueError instead of being ignored. A grid with one cell
in k runs as the 2.5-D step (do25D), the GPU step's form of a single k layer.
"""
from __future__ import annotations

import xml.etree.ElementTree as ET

import numpy as np

from mage_b200 import grids
from mage_b200.gamera import FP64, LIB_PATH, RECON_7UP, RECON_8CENT, GameraGPU, GamParams

HUGE = 1.0e12  # kdefs.F90:20
TINY = 1.0e-12


def read(source: str) -> dict:
    """Keys of the <Kaiju><Gamera> block as {'section/key': value string},
    lower-cased. ``source`` is a path or the XML text itself."""
    text = source if source.lstrip().startswith("<") else open(source).read()
    root = ET.fromstring(text)
    if root.tag.lower() != "kaiju":
        raise ValueError(f"deck root is <{root.tag}>, expected <Kaiju>")
    gam = [e for e in root if e.tag.lower() == "gamera"]
    if not gam:
        raise ValueError("deck has no <Gamera> block")
    out = {}
    for sec in gam[0]:
        for k, v in sec.attrib.items():
            out[f"{sec.tag.lower()}/{k.lower()}"] = v.strip()
    return out


def _bool(s: str) -> bool:
    """Fortran list-directed input of a logical: optional '.', then T or F."""
    t = s.strip().lstrip(".").upper()
    if t[:1] == "T":
        return True
    if t[:1] == "F":
        return False
    raise ValueError(f"not a Fortran logical: {s!r}")


class Deck:
    """The keys of one deck with typed, defaulted access (Set_Val)."""

    def __init__(self, source: str):
        self.kv = read(source)

    def has(self, key: str) -> bool:
        return key.lower() in self.kv

    def bool(self, key: str, default: bool) -> bool:
        v = self.kv.get(key.lower(), "")
        return _bool(v) if v else default

    def float(self, key: str, default: float) -> float:
        v = self.kv.get(key.lower(), "")
        return float(v.replace("d", "e").replace("D", "e")) if v else float(default)

    def int(self, key: str, default: int) -> int:
        v = self.kv.get(key.lower(), "")
        return int(v) if v else int(default)

    def str(self, key: str, default: str) -> str:
        v = self.kv.get(key.lower(), "")
        return v if v else default


_UNSUPPORTED = (("physics/doResistive", "resistivity"), ("multifluid/doMF", "multifluid"),
                ("timestep/doCPR", "CPR"), ("grid/doCyl", "cylindrical grid generation"),
                ("grid/doSph", "spherical grid generation"), ("grid/doWarp", "warped grid generation"),
                ("grid/doStretch", "stretched grid generation"), ("sim/doH5g", "HDF5 grids"),
                ("restart/doRes", "HDF5 restarts"), ("prob/doBz", "the blast wave's Bz option"),
                ("prob/doBack", "the blast wave's background field"))


def params(d: Deck, precision: int = FP64, strict: bool = False) -> GamParams:
    """GamParams from the deck with the reference's defaults."""
    for key, what in _UNSUPPORTED:
        if d.bool(key, False):
            raise ValueError(f"{key} = T: {what} is not part of the GPU step")
    N = [d.int(f"{x}dir/N", 0) for x in "ijk"]
    if min(N) < 1:
        raise ValueError("idir/N, jdir/N and kdir/N must be given")
    pdmb = d.float("sim/pdmb", 0.75)
    C0 = min(0.5 / (pdmb + 0.5), 0.3)
    doHogs = d.bool("physics/doHogs", True)
    doBoris = d.bool("physics/doBoris", False)
    rmeth = d.str("sim/rmeth", "8CENT").upper()
    if rmeth not in ("8CENT", "7UP"):
        raise ValueError(f"sim/rmeth = {rmeth}: the GPU step has 8CENT and 7UP")
    dFloor = d.float("sim/dFloor", TINY)
    dFloor = d.float("floors/dFloor", dFloor)
    pFloor = d.float("sim/pFloor", TINY)
    pFloor = d.float("floors/pFloor", pFloor)
    fixed = d.float("time/fixedTimestep", -1.0)
    if N[1] < 4:
        raise ValueError("jdir/N < 4: the GPU step fills 4 ghost layers from active ones (use N >= 4 for a 1-D problem)")
    gamma0 = 1.4 if d.str("sim/icType", "OT2D").upper() == "ADV1D" else 5.0 / 3.0  # initADV1D, prob.F90:682
    return GamParams(N[0], N[1], N[2], gamma=d.float("physics/gamma", gamma0), CFL=d.float("sim/CFL", C0),
                     pdmb=pdmb, Vd0=d.float("sim/Vd0", 0.5),
                     cHogH=d.float("physics/cHogH", 0.25) if doHogs else 0.0,
                     cHogM=d.float("physics/cHogM", 0.25) if doHogs else 0.0,
                     dFloor=dFloor, pFloor=pFloor, tFin=d.float("time/tFin", 1.0),
                     limDT0=d.float("timestep/limDT0", 1.0e-3), fixedTimestep=fixed if fixed > 0 else -1.0,
                     rmeth=RECON_7UP if rmeth == "7UP" else RECON_8CENT, doLFMLim=d.bool("sim/lfmlim", True),
                     doMHD=d.bool("physics/doMHD", False), do25D=d.bool("physics/do25D", False) or N[2] == 1,
                     precision=precision, strict=strict, doBoris=doBoris,
                     Ca=d.float("physics/Ca", HUGE) if doBoris else HUGE, doAB3=d.bool("sim/doAB3", False))


def corners(d: Deck) -> np.ndarray:
    """Uniform Cartesian corners of idir/jdir/kdir (genGridXML)."""
    N = [d.int(f"{x}dir/N", 0) for x in "ijk"]
    b = []
    for x in "ijk":
        b += [d.float(f"{x}dir/min", 0.0), d.float(f"{x}dir/max", 1.0)]
    return grids.uniform_corners(N[0], N[1], N[2], tuple(b))


def blast_wave_args(d: Deck) -> dict:
    """initBW's prob/ keys (prob.F90:209-228)."""
    for v in ("Vx0", "Vy0", "Vz0"):
        if d.float(f"prob/{v}", 0.0) != 0.0:
            raise ValueError(f"prob/{v} != 0: a moving blast wave is not part of the GPU step's initial conditions")
    return {"x0": d.float("prob/x0", 0.0), "y0": d.float("prob/y0", 0.0), "z0": d.float("prob/z0", 0.0),
            "D0": d.float("prob/D0", 1.0), "P0": d.float("prob/P0", 0.1), "pRat": d.float("prob/pRat", 100.0),
            "dRat": d.float("prob/dRat", 1.0), "rC": d.float("prob/rC", 0.1), "B0": d.float("prob/B0", 1.0)}


# prob/ keys the device set-ups take at the reference's defaults only
_FIXED_PROB = {"ADV2D": {"d0": 1.0, "P0": 1.0, "R0": 0.3, "x0": 0.0, "y0": 0.0},
               "LOOP2D": {"d0": 1.0, "P0": 1.0, "Vz0": 0.0, "A0": 1.0e-3, "R0": 0.3, "x0": 0.0, "y0": 0.0},
               "ALFVEN": {"d0": 1.0, "P0": 0.1, "B_para": 1.0, "V_para": 0.0}}


def load(source: str, precision: int = FP64, strict: bool = False, lib_path: str = LIB_PATH):
    """A GameraGPU handle set up from the deck (grid, initial condition by
    sim/icType) and the deck itself."""
    d = Deck(source)
    ic = d.str("sim/icType", "OT2D").upper()
    if ic not in ("OT2D", "BW", "ADV1D", "ADV2D", "LOOP2D", "ALFVEN"):
        raise ValueError(f"sim/icType = {ic}: not one of the set-ups of the GPU step")
    for k, v in _FIXED_PROB.get(ic, {}).items():
        if d.has(f"prob/{k}") and abs(d.float(f"prob/{k}", v) - v) > 1e-12 * max(1.0, abs(v)):
            raise ValueError(f"prob/{k} = {d.str('prob/' + k, '')}: the GPU set-up of {ic} takes the default {v}")
    g = GameraGPU(params(d, precision, strict), lib_path=lib_path)
    g.set_geometry(corners(d))
    if ic == "OT2D":
        g.init_orszag_tang()
    elif ic == "BW":
        g.init_blast_wave(**blast_wave_args(d))
    elif ic in ("ADV2D", "LOOP2D"):
        g.init_test_problem(ic, d.float("prob/V0", 1.0), d.float("prob/alpha", 60.0))
    elif ic == "ALFVEN":
        g.init_test_problem(ic, d.float("prob/alp", float(np.pi) / 3.0))
    else:
        g.init_test_problem(ic)
    return g, d
