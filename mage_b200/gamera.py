"""Host side of the B200 GAMERA step: ctypes binding of include/gamgpu.h.

Mirrors the reference's app interface for the step (gamApp_T,
src/base/types/gamtypes.F90:301-321): ``init_model`` sets up the Grid and the
State, ``step_gamera`` is ``stepGamera`` (src/gamera/gamapp.F90:73-91) and
``advance_model`` is ``gamApp_T%AdvanceModel`` (src/gamera/gamtypessub.F90:74-90).

Arrays cross the boundary in the reference's Fortran layout: a Fortran array
``A(isg:ieg, jsg:jeg, ksg:keg, 1:nc)`` (i fastest) is a C-ordered numpy
array of shape ``(nc, Nk, Nj, Ni)``; face-centred arrays have ``+1`` in the
three grid dimensions. The CUDA library is required: there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgamgpu.so")
# the same library built with the kernels' index checks and NaN canaries
CHECK_LIB_PATH = os.path.join(HERE, "libgamgpu_check.so")

GAM_OK, GAM_EINVAL, GAM_EBADDIM, GAM_ECUDA, GAM_EDT_BAD, GAM_EDT_DISASTER, GAM_ESTATE, GAM_EHOOK, GAM_EBOUNDS = range(9)
BC_PERIODIC, BC_NONE, BC_ZEROGRAD, BC_SPHIN, BC_WIND, BC_HALO, BC_INFLOW, BC_ION, BC_LFM = 0, 1, 2, 3, 4, 5, 6, 7, 8
RING_PPM, RING_PLM, RING_PCM = 0, 1, 2
RECON_8CENT, RECON_7UP = 0, 1
FP64, FP32 = 0, 1

_ERRNAMES = {1: "GAM_EINVAL", 2: "GAM_EBADDIM", 3: "GAM_ECUDA", 4: "GAM_EDT_BAD", 5: "GAM_EDT_DISASTER",
             6: "GAM_ESTATE", 7: "GAM_EHOOK", 8: "GAM_EBOUNDS"}


class GamError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class ISide(C.Structure):
    """gam_iside: the inflow and wind values and the wind tables (device
    pointers in the form's precision) of the differentiation form's I-side
    boundaries."""
    _fields_ = [("inflow", C.c_double * 8), ("wind", C.c_double * 8), ("wC", C.c_void_p),
                ("wF", C.c_void_p * 3), ("sF", C.c_void_p * 3)]


class _Params(C.Structure):
    _fields_ = [
        ("Nip", C.c_int32), ("Njp", C.c_int32), ("Nkp", C.c_int32), ("nG", C.c_int32),
        ("gamma", C.c_double), ("CFL", C.c_double), ("pdmb", C.c_double), ("Vd0", C.c_double),
        ("cHogH", C.c_double), ("cHogM", C.c_double), ("dFloor", C.c_double), ("pFloor", C.c_double),
        ("tFin", C.c_double), ("dt0", C.c_double), ("limDT0", C.c_double), ("fixedTimestep", C.c_double),
        ("rmeth", C.c_int32), ("doLFMLim", C.c_int32), ("doMHD", C.c_int32), ("doBackground", C.c_int32),
        ("do25D", C.c_int32), ("precision", C.c_int32), ("strict", C.c_int32), ("bc", C.c_int32 * 6),
        ("doBoris", C.c_int32), ("Ca", C.c_double), ("doAB3", C.c_int32),
    ]


EXPORTED = (
    "gam_default_params", "gam_create", "gam_destroy", "gam_last_error", "gam_set_geometry",
    "gam_set_geometry_arrays", "gam_get_geometry_arrays", "gam_upload_state", "gam_download_state", "gam_step",
    "gam_calc_dt", "gam_divb", "gam_totals", "gam_last_step_ms", "gam_advance_model", "gam_init_orszag_tang",
    "gam_init_blast_wave", "gam_profile_step", "gam_totals_noalloc", "gam_set_background", "gam_get_background",
    "gam_set_background_dipole", "gam_set_wind", "gam_set_wind_series", "gam_init_test_problem", "gam_set_inflow",
    "gam_set_ionosphere", "gam_set_oostate", "gam_get_oostate", "gam_bounds_status", "gam_init_dipole_wind", "gam_write_restart", "gam_read_restart",
    "gam_halo_bytes", "gam_halo_pack", "gam_halo_unpack", "gam_init_finish_halo", "gam_set_start", "gam_step_begin",
    "gam_dt_partial", "gam_step_end", "gam_set_slab_edges", "gam_set_stream", "gam_step_begin_dev",
    "gam_dt_partial_dev", "gam_step_end_dev", "gam_step_status", "gam_flux_forward", "gam_flux_adjoint",
    "gam_efield_forward", "gam_efield_adjoint", "gam_predict_stage", "gam_update_stage", "gam_step_work_bytes",
    "gam_step_fwd_save", "gam_step_adj", "gam_iside_fill", "gam_iside_adjoint", "gam_step_fwd_save_iside",
    "gam_step_adj_iside", "gam_tile_halo_bytes", "gam_tile_halo_pack", "gam_tile_halo_unpack",
    "gam_set_tile_edges", "gam_set_rings", "gam_ring_defaults",
)

# Background-field arrays (Grid_T, gamtypes.F90:233-242): name, components;
# all cell-sized with ghosts
BACKGROUND_ARRAYS = (("fcB0", 9), ("bFlux0", 3), ("edgB0", 6), ("B0", 3), ("dpB0", 3))

_libs: dict = {}
_dp = C.POINTER(C.c_double)


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libgamgpu.so (built by __graft_entry__.build() / mage_b200/csrc/Makefile),
    or another build of it (CHECK_LIB_PATH)."""
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise GamError(GAM_ECUDA, f"{path} is missing: build the CUDA library first (make -C mage_b200/csrc)")
    L = C.CDLL(path)
    L.gam_default_params.argtypes = [C.POINTER(_Params), C.c_int32, C.c_int32, C.c_int32]
    L.gam_create.argtypes = [C.POINTER(_Params), C.POINTER(C.c_void_p)]
    L.gam_destroy.argtypes = [C.c_void_p]
    L.gam_last_error.argtypes = [C.c_void_p]
    L.gam_last_error.restype = C.c_char_p
    L.gam_set_geometry.argtypes = [C.c_void_p, _dp]
    L.gam_set_geometry_arrays.argtypes = [C.c_void_p] + [_dp] * 11
    L.gam_get_geometry_arrays.argtypes = [C.c_void_p] + [_dp] * 11
    L.gam_upload_state.argtypes = [C.c_void_p] + [_dp] * 5 + [C.c_double, C.c_double, C.c_double, C.c_int32]
    L.gam_download_state.argtypes = [C.c_void_p] + [_dp] * 5 + [_dp, _dp, _dp, C.POINTER(C.c_int32)]
    L.gam_step.argtypes = [C.c_void_p, C.c_int32, _dp, _dp]
    L.gam_calc_dt.argtypes = [C.c_void_p, _dp]
    L.gam_divb.argtypes = [C.c_void_p, _dp]
    L.gam_totals.argtypes = [C.c_void_p, _dp]
    L.gam_last_step_ms.argtypes = [C.c_void_p, _dp]
    L.gam_advance_model.argtypes = [C.c_void_p, C.c_double, _dp]
    L.gam_init_orszag_tang.argtypes = [C.c_void_p]
    L.gam_init_blast_wave.argtypes = [C.c_void_p, _dp]
    L.gam_profile_step.argtypes = [C.c_void_p, C.c_int32, _dp, C.c_int32]
    L.gam_set_background.argtypes = [C.c_void_p] + [_dp] * 5
    L.gam_get_background.argtypes = [C.c_void_p] + [_dp] * 5
    L.gam_set_background_dipole.argtypes = [C.c_void_p, C.c_double]
    L.gam_set_wind.argtypes = [C.c_void_p, _dp]
    L.gam_set_inflow.argtypes = [C.c_void_p, _dp]
    L.gam_set_ionosphere.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_double]
    L.gam_set_rings.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.c_int32,
                                C.c_int32]
    L.gam_ring_defaults.argtypes = [C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.gam_init_test_problem.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_double]
    L.gam_set_wind_series.argtypes = [C.c_void_p, C.c_int32] + [_dp] * 6 + [C.c_double] * 3
    L.gam_set_oostate.argtypes = [C.c_void_p, _dp, C.c_double]
    L.gam_get_oostate.argtypes = [C.c_void_p, _dp, _dp]
    L.gam_write_restart.argtypes = [C.c_void_p, C.c_char_p]
    L.gam_halo_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.gam_set_slab_edges.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    L.gam_set_tile_edges.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
    L.gam_tile_halo_bytes.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]
    L.gam_tile_halo_pack.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]
    L.gam_tile_halo_unpack.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32]
    L.gam_flux_forward.argtypes = [C.POINTER(_Params), C.c_int32] + [C.c_void_p] * 8 + [_dp, _dp] + [C.c_void_p] * 3
    L.gam_flux_adjoint.argtypes = [C.POINTER(_Params), C.c_int32] + [C.c_void_p] * 8 + [_dp, _dp] + [C.c_void_p] * 8
    L.gam_efield_forward.argtypes = [C.POINTER(_Params), C.c_int32] + [C.c_void_p] * 9 + [_dp, C.c_double] + \
        [C.c_void_p] * 3
    L.gam_efield_adjoint.argtypes = [C.POINTER(_Params), C.c_int32] + [C.c_void_p] * 9 + [_dp, C.c_double] + \
        [C.c_void_p] * 8
    _vpp = C.POINTER(C.c_void_p)
    L.gam_predict_stage.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _vpp, C.c_double, C.c_double, _vpp, _vpp,
                                    C.c_void_p, _vpp, C.c_void_p]
    L.gam_update_stage.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _vpp, _dp, C.c_double, _vpp, _vpp,
                                   C.c_void_p, C.c_void_p, _vpp, C.c_void_p]
    L.gam_step_work_bytes.argtypes = [C.POINTER(_Params), C.c_int32, C.POINTER(C.c_int64)]
    L.gam_step_fwd_save.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _vpp, _vpp, C.c_double, C.c_double, _vpp,
                                    C.c_void_p, C.c_void_p]
    L.gam_step_adj.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _vpp, _vpp, C.c_double, C.c_double, C.c_int32,
                               _vpp, _vpp, C.c_void_p, C.c_void_p]
    _isp = C.POINTER(ISide)
    L.gam_iside_fill.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _isp, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p]
    L.gam_iside_adjoint.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _isp] + [C.c_void_p] * 7
    L.gam_step_fwd_save_iside.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _vpp, _isp, _vpp, C.c_double,
                                          C.c_double, _vpp, C.c_void_p, C.c_void_p]
    L.gam_step_adj_iside.argtypes = [C.POINTER(_Params), C.c_int32, _vpp, _vpp, _isp, _vpp, C.c_double, C.c_double,
                                     C.c_int32, _vpp, _vpp, C.c_void_p, C.c_void_p, C.c_void_p]
    L.gam_halo_pack.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    L.gam_halo_unpack.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
    L.gam_init_finish_halo.argtypes = [C.c_void_p, _dp]
    L.gam_set_start.argtypes = [C.c_void_p, C.c_double]
    L.gam_step_begin.argtypes = [C.c_void_p]
    L.gam_dt_partial.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]
    L.gam_step_end.argtypes = [C.c_void_p, C.c_uint64, C.c_int32, _dp, _dp]
    L.gam_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.gam_step_begin_dev.argtypes = [C.c_void_p]
    L.gam_dt_partial_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.gam_step_end_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.gam_step_status.argtypes = [C.c_void_p, _dp, _dp]
    L.gam_read_restart.argtypes = [C.c_void_p, C.c_char_p]
    L.gam_init_dipole_wind.argtypes = [C.c_void_p, _dp, C.c_uint64, C.c_double]
    L.gam_totals_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                     C.c_void_p, C.c_char_p, C.c_int32]
    L.gam_bounds_status.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    _libs[path] = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


@dataclass
class GamParams:
    """Model keys of the step; defaults are the reference's (init.F90:312-484)."""
    Nip: int
    Njp: int
    Nkp: int
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
    fixedTimestep: float = -1.0
    rmeth: int = RECON_8CENT
    doLFMLim: bool = True
    doMHD: bool = True
    doBackground: bool = False
    do25D: bool = False
    precision: int = FP64
    strict: bool = False
    bc: tuple = field(default_factory=lambda: (BC_PERIODIC,) * 6)
    doBoris: bool = False
    Ca: float = 1.0e12
    doAB3: bool = False

    def to_c(self) -> _Params:
        p = _Params()
        p.nG = 4
        for f, _ in _Params._fields_:
            if f == "nG":
                continue
            if f == "bc":
                p.bc[:] = list(self.bc)
            else:
                setattr(p, f, getattr(self, f))
        return p

    @property
    def dims(self):
        return self.Nip + 8, self.Njp + 8, self.Nkp + 8


GEOMETRY_ARRAYS = (("face", "face", 3), ("xfc", "face", 9), ("Tf", "face", 27), ("volume", "cell", 1),
                   ("xyzcc", "cell", 3), ("di", "cell", 1), ("dj", "cell", 1), ("dk", "cell", 1),
                   ("edge", "face", 3), ("Te", "face", 27), ("Teb", "face", 12))


def ring_defaults(Np: int, aggressive: bool = False, lib_path: str = LIB_PATH) -> list:
    """The reference's default chunks per ring for Np cells around the LFM axis."""
    L = load_library(lib_path)
    n = C.c_int32()
    a = (C.c_int32 * 32)()
    rc = L.gam_ring_defaults(int(Np), int(bool(aggressive)), C.byref(n), a)
    if rc:
        raise GamError(rc, f"no default rings for Np = {Np}")
    return [int(a[q]) for q in range(n.value)]


class GameraGPU:
    """One GAMERA app whose Grid and State live on the GPU."""

    def __init__(self, params: GamParams, lib_path: str = LIB_PATH):
        self.L = load_library(lib_path)
        self._lib_path = lib_path
        self.params = params
        self._cp = params.to_c()
        h = C.c_void_p()
        rc = self.L.gam_create(C.byref(self._cp), C.byref(h))
        self.h = h
        self._check(rc)
        self.Ni, self.Nj, self.Nk = params.dims

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            self.L.gam_destroy(h)
            self.h = None

    def close(self):
        self.__del__()

    def _check(self, rc: int):
        if rc != GAM_OK:
            msg = self.L.gam_last_error(self.h).decode() if self.h and self.h.value else ""
            raise GamError(rc, msg)

    def shape(self, kind: str, nc: int):
        if kind == "cell":
            return (nc, self.Nk, self.Nj, self.Ni)
        return (nc, self.Nk + 1, self.Nj + 1, self.Ni + 1)

    # --- grid ---------------------------------------------------------------
    def set_geometry(self, xyz: np.ndarray):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        assert xyz.shape == self.shape("face", 3), xyz.shape
        self._check(self.L.gam_set_geometry(self.h, _ptr(xyz)))

    def set_geometry_arrays(self, arrs: dict):
        args = []
        keep = []
        for name, kind, nc in GEOMETRY_ARRAYS:
            a = np.ascontiguousarray(arrs[name], dtype=np.float64).reshape(self.shape(kind, nc))
            keep.append(a)
            args.append(_ptr(a))
        self._check(self.L.gam_set_geometry_arrays(self.h, *args))

    def get_geometry_arrays(self) -> dict:
        out = {name: np.zeros(self.shape(kind, nc)) for name, kind, nc in GEOMETRY_ARRAYS}
        self._check(self.L.gam_get_geometry_arrays(self.h, *[_ptr(out[n]) for n, _, _ in GEOMETRY_ARRAYS]))
        return out

    # --- state --------------------------------------------------------------
    def upload_state(self, Gas, magFlux, Bxyz, oGas, omagFlux, time: float, otime: float, dt: float, ts: int = 0):
        """oGas = omagFlux = None: oState stays on the device (after a step it is
        the State before that step); only State is copied. Bxyz = None: computed
        from magFlux on the device (bFlux2Fld)."""
        keep_old = oGas is None and omagFlux is None
        src = (Gas, magFlux, Bxyz) if keep_old else (Gas, magFlux, Bxyz, oGas, omagFlux)
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in src]
        shapes = [self.shape("cell", 5), self.shape("face", 3), self.shape("cell", 3), self.shape("cell", 5),
                  self.shape("face", 3)]
        for a, s in zip(arrs, shapes):
            assert a is None or a.shape == s, (a.shape, s)
        ptrs = [None if a is None else _ptr(a) for a in arrs] + ([None, None] if keep_old else [])
        self._check(self.L.gam_upload_state(self.h, *ptrs, time, otime, dt, int(ts)))

    def set_oostate(self, oomagFlux, ootime: float):
        """ooState face fluxes and time of the AB3 predictor (doAB3)."""
        a = np.ascontiguousarray(oomagFlux, dtype=np.float64)
        assert a.shape == self.shape("face", 3), a.shape
        self._check(self.L.gam_set_oostate(self.h, _ptr(a), float(ootime)))

    def bounds_status(self) -> dict:
        """Record of the bounds-check build: fired 1 / 0, or -1 without checks."""
        f, k, i = C.c_int32(), C.c_int32(), C.c_int64()
        self._check(self.L.gam_bounds_status(self.h, C.byref(f), C.byref(k), C.byref(i)))
        return {"fired": f.value, "kernel": k.value, "index": i.value}

    def get_oostate(self) -> dict:
        a = np.zeros(self.shape("face", 3))
        t = C.c_double()
        self._check(self.L.gam_get_oostate(self.h, _ptr(a), C.byref(t)))
        return {"oomagFlux": a, "ootime": t.value}

    def download_state(self, into: dict | None = None, old: bool = True, names=None) -> dict:
        """State (and with ``old`` the previous state) in Fortran layout;
        ``into`` may supply preallocated (e.g. pinned) arrays; ``names`` picks
        the arrays (the others are not copied)."""
        if names is None:
            names = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux") if old else ("Gas", "magFlux", "Bxyz")
        kinds = {"Gas": ("cell", 5), "magFlux": ("face", 3), "Bxyz": ("cell", 3), "oGas": ("cell", 5),
                 "omagFlux": ("face", 3)}
        out = {}
        for k in names:
            a = into.get(k) if into else None
            if a is None:
                a = np.zeros(self.shape(*kinds[k]))
            assert a.shape == self.shape(*kinds[k]) and a.dtype == np.float64 and a.flags.c_contiguous
            out[k] = a
        ptrs = [(_ptr(out[k]) if k in out else None) for k in ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")]
        t, ot, dt, ts = C.c_double(), C.c_double(), C.c_double(), C.c_int32()
        self._check(self.L.gam_download_state(self.h, *ptrs, C.byref(t), C.byref(ot), C.byref(dt), C.byref(ts)))
        out.update(time=t.value, otime=ot.value, dt=dt.value, ts=ts.value)
        return out

    # --- problems -------------------------------------------------------------
    def init_orszag_tang(self):
        self._check(self.L.gam_init_orszag_tang(self.h))

    TEST_PROBLEMS = {"ADV1D": 2, "ADV2D": 3, "LOOP2D": 4, "ALFVEN": 5}

    def init_test_problem(self, name: str, a: float = 0.0, b: float = 0.0):
        """initADV1D / initADV2D (a = V0, b = alpha) / initLoop (a = V0, b = alpha) /
        initALFVEN (a = alp) of prob.F90."""
        self._check(self.L.gam_init_test_problem(self.h, self.TEST_PROBLEMS[name.upper()], float(a), float(b)))

    def init_blast_wave(self, x0=0.5, y0=0.5, z0=0.5, D0=1.0, P0=0.1, pRat=100.0, dRat=1.0, rC=0.1, B0=1.0):
        bw = np.array([x0, y0, z0, D0, P0, pRat, dRat, rC, B0], dtype=np.float64)
        self._check(self.L.gam_init_blast_wave(self.h, _ptr(bw)))

    # --- background field and solar wind --------------------------------------
    def set_background(self, arrs: dict):
        """Upload fcB0, bFlux0, edgB0, B0, dpB0 (Fortran layout, cell-sized)."""
        keep = [np.ascontiguousarray(arrs[n], dtype=np.float64).reshape(self.shape("cell", nc))
                for n, nc in BACKGROUND_ARRAYS]
        self._check(self.L.gam_set_background(self.h, *[_ptr(a) for a in keep]))

    def get_background(self) -> dict:
        out = {n: np.zeros(self.shape("cell", nc)) for n, nc in BACKGROUND_ARRAYS}
        self._check(self.L.gam_get_background(self.h, *[_ptr(out[n]) for n, _ in BACKGROUND_ARRAYS]))
        return out

    def set_background_dipole(self, M0: float):
        """AddB0 on the device for the dipole of moment (0, 0, M0)."""
        self._check(self.L.gam_set_background_dipole(self.h, float(M0)))

    def set_wind(self, wind):
        """Constant solar wind {rho, P, Vx, Vy, Vz, Bx, By, Bz} of the outer-I boundary."""
        w = np.ascontiguousarray(wind, dtype=np.float64)
        assert w.shape == (8,)
        self._check(self.L.gam_set_wind(self.h, _ptr(w)))

    def set_wind_series(self, t, rho, P, V, B, xyzBS=None, Bx0=0.0, ByC=0.0, BzC=0.0):
        """Solar-wind time series of the outer-I boundary (code units); V, B, xyzBS are (n, 3)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (t, rho, P, V, B)]
        xb = None if xyzBS is None else np.ascontiguousarray(xyzBS, dtype=np.float64)
        n = arrs[0].size
        assert arrs[1].size == n and arrs[2].size == n and arrs[3].shape == (n, 3) and arrs[4].shape == (n, 3)
        self._check(self.L.gam_set_wind_series(self.h, n, *[_ptr(a) for a in arrs], None if xb is None else _ptr(xb),
                                               float(Bx0), float(ByC), float(BzC)))

    def set_inflow(self, state):
        """Uniform inner-I inflow {rho, P, Vx, Vy, Vz, Bx, By, Bz} (bc[0] = BC_INFLOW)."""
        w = np.ascontiguousarray(state, dtype=np.float64)
        assert w.shape == (8,)
        self._check(self.L.gam_set_inflow(self.h, _ptr(w)))

    def set_rings(self, Nch=None, recon: int = RING_PPM, nft: int = 1, clean: bool = True, fast_clean: bool = True):
        """Ring averaging about the LFM axis (bc[2] / bc[3] = BC_LFM), before
        the geometry: chunks per ring (default: the reference's table for
        Nkp), ring reconstruction, Fourier modes removed from the fluxes,
        CleanLoops and its fast form."""
        if Nch is None:
            Nch = ring_defaults(self.params.Nkp, lib_path=self._lib_path)
        a = (C.c_int32 * 32)(*[int(x) for x in Nch])
        self._check(self.L.gam_set_rings(self.h, len(Nch), a, int(recon), int(nft), int(bool(clean)),
                                         int(bool(fast_clean))))

    def set_ionosphere(self, inExyz, inEijk, M0: float, dtCpl: float = 0.0, doIonPush: bool = True, nIonP: int = 1,
                       dtSW0: float = 60.0 / 63.8):
        """Coupling fields of the ionospheric inner boundary (bc[0] = BC_ION):
        inExyz (3, Nk+8, Nj+8, 5) and inEijk (3, Nk+9, Nj+9, 6) in C order,
        i.e. the Fortran arrays (1:5, jsg:jeg, ksg:keg, 1:3) and
        (1:6, jsg:jeg+1, ksg:keg+1, 1:3); M0 the dipole moment; dtCpl the
        coupling time scale of PushIon and dtSW0 that of NudgeSW (code time;
        60 s in Earth units, the reference's one minute, is the default).
        A tile away from the inner boundary (bc[0] = BC_HALO) passes None for
        both fields: it takes the hooks of its other sides and the DT range."""
        if inExyz is None:
            E = Ee = None
            pE = pEe = None
        else:
            E = np.ascontiguousarray(inExyz, dtype=np.float64)
            Ee = np.ascontiguousarray(inEijk, dtype=np.float64)
            pE, pEe = _ptr(E), _ptr(Ee)
        self._check(self.L.gam_set_ionosphere(self.h, pE, pEe, float(M0), float(dtCpl),
                                              int(bool(doIonPush)), int(nIonP), float(dtSW0)))

    def init_dipole_wind(self, wind, seed: int = 31337, amp: float = 0.01):
        """Wind state with a seeded density perturbation and the wind's uniform field."""
        w = np.ascontiguousarray(wind, dtype=np.float64)
        assert w.shape == (8,)
        self._check(self.L.gam_init_dipole_wind(self.h, _ptr(w), int(seed), float(amp)))

    # --- tiling (see mage_b200.tiling) ---------------------------------------------
    def set_slab_edges(self, lowest: bool, highest: bool):
        self._check(self.L.gam_set_slab_edges(self.h, int(lowest), int(highest)))

    def set_tile_edges(self, d: int, lowest: bool, highest: bool):
        """Whether this tile's lower / upper side in direction d (0 I, 1 J,
        2 K) is an edge of the whole grid (CalcDT's ghost layer)."""
        self._check(self.L.gam_set_tile_edges(self.h, int(d), int(lowest), int(highest)))

    def tile_halo_bytes(self, d: int) -> int:
        n = C.c_int64()
        self._check(self.L.gam_tile_halo_bytes(self.h, int(d), C.byref(n)))
        return n.value

    def tile_halo_pack(self, d: int, side: int, buf):
        """Pack the halo of side 0 (down) or 1 (up) of direction d into a
        device buffer (a tensor or a pointer)."""
        ptr = buf.data_ptr() if hasattr(buf, "data_ptr") else int(buf)
        self._check(self.L.gam_tile_halo_pack(self.h, int(d), int(side), C.c_void_p(ptr)))

    def tile_halo_unpack(self, d: int, side: int, buf, copyB: bool = False):
        ptr = buf.data_ptr() if hasattr(buf, "data_ptr") else int(buf)
        self._check(self.L.gam_tile_halo_unpack(self.h, int(d), int(side), C.c_void_p(ptr), int(copyB)))

    def halo_bytes(self) -> int:
        n = C.c_int64()
        self._check(self.L.gam_halo_bytes(self.h, C.byref(n)))
        return n.value

    def halo_pack(self, side: int, buf):
        """Pack side 0 (down) or 1 (up) into a device buffer (a tensor or a pointer)."""
        ptr = buf.data_ptr() if hasattr(buf, "data_ptr") else int(buf)
        self._check(self.L.gam_halo_pack(self.h, int(side), C.c_void_p(ptr)))

    def halo_unpack(self, side: int, buf, copyB: bool = False):
        ptr = buf.data_ptr() if hasattr(buf, "data_ptr") else int(buf)
        self._check(self.L.gam_halo_unpack(self.h, int(side), C.c_void_p(ptr), int(copyB)))

    def init_finish_halo(self) -> float:
        dt = C.c_double()
        self._check(self.L.gam_init_finish_halo(self.h, C.byref(dt)))
        return dt.value

    def set_start(self, dt: float):
        self._check(self.L.gam_set_start(self.h, float(dt)))

    def step_begin(self):
        self._check(self.L.gam_step_begin(self.h))

    def dt_partial(self):
        bits, nbad = C.c_uint64(), C.c_int32()
        self._check(self.L.gam_dt_partial(self.h, C.byref(bits), C.byref(nbad)))
        return bits.value, nbad.value

    def step_end(self, bits: int, nbad: int):
        dt, t = C.c_double(), C.c_double()
        self._check(self.L.gam_step_end(self.h, C.c_uint64(bits), int(nbad), C.byref(dt), C.byref(t)))
        return dt.value, t.value

    # device-resident tile steps (no host round trip per step)
    def set_stream(self, stream_ptr: int | None):
        """Enqueue this handle's work on the caller's CUDA stream (a
        non-default stream; None: the handle's own)."""
        self._check(self.L.gam_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def step_begin_dev(self):
        self._check(self.L.gam_step_begin_dev(self.h))

    def dt_partial_dev(self, bits, nbad):
        """Write this slab's dt candidate bits and bad-cell count into the
        one-element int64 device tensors bits and nbad."""
        self._check(self.L.gam_dt_partial_dev(self.h, C.c_void_p(bits.data_ptr()), C.c_void_p(nbad.data_ptr())))

    def step_end_dev(self, bits, nbad):
        """Finish the step with the reduced values in device tensors bits, nbad."""
        self._check(self.L.gam_step_end_dev(self.h, C.c_void_p(bits.data_ptr()), C.c_void_p(nbad.data_ptr())))

    def step_status(self):
        """Wait for the handle's stream; (dt, t) after the last step, raising
        GamError if one of the steps since the previous check failed."""
        dt, t = C.c_double(), C.c_double()
        self._check(self.L.gam_step_status(self.h, C.byref(dt), C.byref(t)))
        return dt.value, t.value

    # --- restart files --------------------------------------------------------
    def write_restart(self, path: str):
        """State, oState, times, ts, dt and dt0 to a binary restart file."""
        self._check(self.L.gam_write_restart(self.h, os.fsencode(path)))

    def read_restart(self, path: str):
        """Load a restart file written by write_restart (same grid size)."""
        self._check(self.L.gam_read_restart(self.h, os.fsencode(path)))

    # --- stepping -------------------------------------------------------------
    def step_gamera(self, n: int = 1):
        """n x stepGamera; returns (Model%dt, Model%t)."""
        dt, t = C.c_double(), C.c_double()
        self._check(self.L.gam_step(self.h, int(n), C.byref(dt), C.byref(t)))
        return dt.value, t.value

    def advance_model(self, dt: float) -> float:
        t = C.c_double()
        self._check(self.L.gam_advance_model(self.h, float(dt), C.byref(t)))
        return t.value

    def calc_dt(self) -> float:
        dt = C.c_double()
        self._check(self.L.gam_calc_dt(self.h, C.byref(dt)))
        return dt.value

    def divb(self) -> float:
        v = C.c_double()
        self._check(self.L.gam_divb(self.h, C.byref(v)))
        return v.value

    def totals(self) -> np.ndarray:
        out = np.zeros(5)
        self._check(self.L.gam_totals(self.h, _ptr(out)))
        return out

    KERNEL_NAMES = ("begin", "predict", "mom2face_i", "vxb_i", "mom2face_j", "vxb_j", "mom2face_k", "vxb_k",
                    "stress_i", "stress_j", "stress_k", "update_faces", "update_cells", "dt_finalize", "bc")

    def profile_step(self, reps: int = 5) -> dict:
        """Device time (ms) of each kernel of one step (diagnostic)."""
        ms = np.zeros(15)
        self._check(self.L.gam_profile_step(self.h, int(reps), _ptr(ms), 15))
        return dict(zip(self.KERNEL_NAMES, ms.tolist()))

    def last_step_ms(self) -> float:
        v = C.c_double()
        self._check(self.L.gam_last_step_ms(self.h, C.byref(v)))
        return v.value
