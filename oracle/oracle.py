"""ctypes front end of the CPU restatement of the GAMERA step (oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker. The product never imports it.

Arrays are exposed as numpy views in the reference's memory layout (Fortran
column-major, i fastest): a Fortran array ``A(isg:ieg, jsg:jeg, ksg:keg, 1:nc)``
is a C-ordered numpy array of shape ``(nc, Nk, Nj, Ni)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
VARIANTS = ("strict", "gm", "fast")

BC_PERIODIC = 0
BC_NONE = 1
BC_ZEROGRAD = 2
BC_SPHIN = 3
BC_WIND = 4
BC_INFLOW = 6
BC_ION = 7
BC_LFM = 8


def build(quiet: bool = True) -> None:
    """Compile the three oracle variants (oracle/Makefile)."""
    subprocess.run(["make", "-C", HERE, "-j3"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


class _Params(C.Structure):
    _fields_ = [
        ("Nip", C.c_int), ("Njp", C.c_int), ("Nkp", C.c_int),
        ("doMHD", C.c_int), ("doLFMLim", C.c_int), ("do25D", C.c_int),
        ("doBackground", C.c_int), ("up7", C.c_int), ("fixedTimestep", C.c_int),
        ("gamma", C.c_double), ("CFL", C.c_double), ("pdmb", C.c_double), ("Vd0", C.c_double),
        ("cHogH", C.c_double), ("cHogM", C.c_double), ("dFloor", C.c_double), ("pFloor", C.c_double),
        ("tFin", C.c_double), ("dt0", C.c_double), ("limDT0", C.c_double), ("fixedDT", C.c_double),
        ("bc", C.c_int * 6), ("noMetric", C.c_int), ("M0", C.c_double), ("wind", C.c_double * 8),
        ("inflow", C.c_double * 8), ("doBoris", C.c_int), ("Ca", C.c_double),
        ("doAB3", C.c_int), ("ringNumR", C.c_int), ("ringNch", C.c_int * 32), ("ringRecon", C.c_int),
        ("ringNFT", C.c_int), ("ringClean", C.c_int), ("ringFast", C.c_int),
    ]


class _Scalars(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("dt0", C.c_double),
                ("time", C.c_double), ("otime", C.c_double), ("ts", C.c_int), ("status", C.c_int),
                ("ootime", C.c_double)]


@dataclass
class OracleParams:
    """Model keys of the step (init.F90:312-484 defaults unless stated)."""
    Nip: int
    Njp: int
    Nkp: int
    doMHD: bool = True
    doLFMLim: bool = True
    do25D: bool = False
    doBackground: bool = False
    up7: bool = False
    fixedTimestep: bool = False
    gamma: float = 5.0 / 3.0
    CFL: float = 0.3
    pdmb: float = 0.75
    Vd0: float = 0.5
    cHogH: float = 0.25
    cHogM: float = 0.25
    dFloor: float = 1.0e-12
    pFloor: float = 1.0e-12
    tFin: float = 1.0e30
    dt0: float = 0.0
    limDT0: float = 1.0e-3
    fixedDT: float = 0.0
    bc: tuple = field(default_factory=lambda: (BC_PERIODIC,) * 6)
    noMetric: bool = False
    M0: float = 0.0
    wind: tuple = (0.0,) * 8
    inflow: tuple = (0.0,) * 8
    doBoris: bool = False
    Ca: float = 0.0
    doAB3: bool = False
    # ring averaging about the LFM axis: chunks per ring (empty: off), ring
    # reconstruction (0 PPM, 1 PLM, 2 PCM), Fourier modes removed from the
    # fluxes, loop cleaning and its fast form
    ringNch: tuple = ()
    ringRecon: int = 0
    ringNFT: int = 1
    ringClean: bool = True
    ringFast: bool = True

    def to_c(self) -> _Params:
        p = _Params()
        for f, _ in _Params._fields_:
            if f == "bc":
                p.bc[:] = list(self.bc)
            elif f == "ringNumR":
                p.ringNumR = len(self.ringNch)
            elif f == "ringNch":
                p.ringNch[:len(self.ringNch)] = list(self.ringNch)
            elif f in ("wind", "inflow"):
                getattr(p, f)[:] = list(getattr(self, f))
            else:
                setattr(p, f, getattr(self, f))
        return p


_ARR = {"Gas": (0, "cell", 5), "magFlux": (1, "face", 3), "Bxyz": (2, "cell", 3),
        "oGas": (3, "cell", 5), "omagFlux": (4, "face", 3), "oBxyz": (5, "cell", 3),
        "xyzcc": (6, "cell", 3), "xfc": (7, "face", 9), "volume": (8, "cell", 1),
        "di": (9, "cell", 1), "dj": (10, "cell", 1), "dk": (11, "cell", 1),
        "Tf": (12, "face", 27), "Te": (13, "face", 27), "Teb": (14, "face", 12),
        "face": (15, "face", 3), "edge": (16, "face", 3), "Efld": (17, "cell", 3),
        "hGas": (18, "cell", 5), "hmagFlux": (19, "face", 3), "hBxyz": (20, "cell", 3),
        "dGasH": (21, "cell", 5), "dGasM": (22, "cell", 3), "xyz": (23, "face", 3),
        "fcB0": (24, "cell", 9), "bFlux0": (25, "cell", 3), "edgB0": (26, "cell", 6), "B0": (27, "cell", 3),
        "dpB0": (28, "cell", 3), "ooGas": (29, "cell", 5), "oomagFlux": (30, "face", 3), "ooBxyz": (31, "cell", 3)}

_libs: dict = {}


def lib(variant: str = "strict") -> C.CDLL:
    if variant not in _libs:
        path = os.path.join(BUILD, f"liborc_{variant}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(_Params), C.POINTER(C.c_double)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_array.restype = C.POINTER(C.c_double)
        L.orc_array.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_long)]
        L.orc_ic_ot.argtypes = [C.c_void_p]
        L.orc_ic_bw.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_ic_dipole_wind.argtypes = [C.c_void_p, C.c_double, C.c_ulonglong]
        L.orc_set_background_noalloc.argtypes = [C.c_void_p]
        L.orc_init_finish.argtypes = [C.c_void_p]
        L.orc_init_finish.restype = C.c_int
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_step.restype = C.c_int
        L.orc_scalars.argtypes = [C.c_void_p, C.POINTER(_Scalars)]
        L.orc_set_scalars.argtypes = [C.c_void_p, C.POINTER(_Scalars)]
        L.orc_divb.argtypes = [C.c_void_p]
        L.orc_divb.restype = C.c_double
        L.orc_ring_average.argtypes = [C.c_void_p]
        L.orc_ring_average.restype = C.c_int
        for f in ("orc_c2p", "orc_p2c"):
            getattr(L, f).argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        for f in ("orc_erfc", "orc_exp"):
            getattr(L, f).argtypes = [C.c_double]
            getattr(L, f).restype = C.c_double
        L.orc_num_threads.restype = C.c_int
        L.orc_ic_case.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.orc_set_wind_series.argtypes = [C.c_void_p, C.c_int] + [C.POINTER(C.c_double)] * 6 + [C.c_double] * 3
        L.orc_set_ionosphere.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                         C.c_double, C.c_int, C.c_int, C.c_double]
        _libs[variant] = L
    return _libs[variant]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One GAMERA app (Model, Grid, State, oState, StateHf) on the CPU."""

    def __init__(self, params: OracleParams, xyz: np.ndarray, variant: str = "strict"):
        self.p = params
        self.L = lib(variant)
        self.Ni, self.Nj, self.Nk = params.Nip + 8, params.Njp + 8, params.Nkp + 8
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        assert xyz.shape == (3, self.Nk + 1, self.Nj + 1, self.Ni + 1), xyz.shape
        self._cp = params.to_c()
        self.h = self.L.orc_create(C.byref(self._cp), _dptr(xyz))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.orc_destroy(h)
            self.h = None

    def array(self, name: str) -> np.ndarray:
        """Live numpy view of an internal array, shape (nc, Nk', Nj', Ni')."""
        which, kind, nc = _ARR[name]
        n = C.c_long()
        ptr = self.L.orc_array(self.h, which, C.byref(n))
        sh = (self.Nk, self.Nj, self.Ni) if kind == "cell" else (self.Nk + 1, self.Nj + 1, self.Ni + 1)
        a = np.ctypeslib.as_array(ptr, shape=(n.value,))
        return a.reshape((nc,) + sh)

    def ic_orszag_tang(self):
        self.L.orc_ic_ot(self.h)

    def ic_blast_wave(self, x0=0.5, y0=0.5, z0=0.5, D0=1.0, P0=0.1, pRat=100.0, dRat=1.0, rC=0.1, B0=1.0):
        a = np.array([x0, y0, z0, D0, P0, pRat, dRat, rC, B0], dtype=np.float64)
        self.L.orc_ic_bw(self.h, _dptr(a))

    def ic_dipole_wind(self, amp: float = 0.01, seed: int = 31337):
        self.L.orc_ic_dipole_wind(self.h, amp, seed)

    def alloc_background(self):
        self.L.orc_set_background_noalloc(self.h)

    def init_finish(self) -> int:
        return self.L.orc_init_finish(self.h)

    def step(self, n: int = 1) -> int:
        return self.L.orc_step(self.h, int(n))

    def scalars(self) -> dict:
        s = _Scalars()
        self.L.orc_scalars(self.h, C.byref(s))
        return {f: getattr(s, f) for f, _ in _Scalars._fields_}

    def set_scalars(self, **kw):
        s = _Scalars()
        self.L.orc_scalars(self.h, C.byref(s))
        for k, v in kw.items():
            setattr(s, k, v)
        self.L.orc_set_scalars(self.h, C.byref(s))

    def ic_case(self, name: str, a: float = 0.0, b: float = 0.0):
        """The reference's test problems (prob.F90): 'adv1d'; 'adv2d' and 'loop2d'
        with a = V0, b = alpha (degrees); 'alfven' with a = alp (radians)."""
        self.L.orc_ic_case(self.h, {"adv1d": 0, "adv2d": 1, "loop2d": 2, "alfven": 3}[name], a, b)

    def set_wind_series(self, t, rho, P, V, B, xyzBS=None, Bx0=0.0, ByC=0.0, BzC=0.0):
        """Solar-wind time series of the outer-I wind boundary (code units)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (t, rho, P, V, B)]
        xb = None if xyzBS is None else np.ascontiguousarray(xyzBS, dtype=np.float64)
        self._ws = arrs + [xb]
        self.L.orc_set_wind_series(self.h, len(arrs[0]), *[_dptr(a) for a in arrs], None if xb is None else _dptr(xb),
                                   Bx0, ByC, BzC)

    def set_ionosphere(self, inExyz, inEijk, M0: float, dtCpl: float, doIonPush: bool = True, nIonP: int = 1,
                       dtSW0: float = 60.0 / 63.8):
        """Coupling fields of the ionospheric inner boundary (bc[0] = 7):
        inExyz (3, Nk+8, Nj+8, 5) and inEijk (3, Nk+9, Nj+9, 6), the C-order
        views of the Fortran arrays (1:5, jsg:jeg, ksg:keg, 1:3) and
        (1:6, jsg:jeg+1, ksg:keg+1, 1:3); dtSW0 NudgeSW's time scale (code
        time; the reference's one minute in Earth units)."""
        self._ionE = np.ascontiguousarray(inExyz, dtype=np.float64)
        self._ionEe = np.ascontiguousarray(inEijk, dtype=np.float64)
        self.L.orc_set_ionosphere(self.h, _dptr(self._ionE), _dptr(self._ionEe), float(M0), float(dtCpl),
                                  int(bool(doIonPush)), int(nIonP), float(dtSW0))

    def divb(self) -> float:
        return self.L.orc_divb(self.h)

    def ring_average(self) -> int:
        """RingAverage alone on the current state (ringav.F90:26-75)."""
        return self.L.orc_ring_average(self.h)


def c2p(con, gamma=5.0 / 3.0, variant="strict"):
    con = np.asarray(con, dtype=np.float64)
    out = np.zeros(5)
    lib(variant).orc_c2p(gamma, _dptr(con), _dptr(out))
    return out


def p2c(prim, gamma=5.0 / 3.0, variant="strict"):
    prim = np.asarray(prim, dtype=np.float64)
    out = np.zeros(5)
    lib(variant).orc_p2c(gamma, _dptr(prim), _dptr(out))
    return out
