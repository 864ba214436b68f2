"""Shared set-up for the parity tests: an oracle app (CPU restatement) and a
GPU app fed with the oracle's metric and initial state through the C ABI,
the way the Fortran driver would feed it."""
import numpy as np

from mage_b200 import grids
from mage_b200.gamera import LIB_PATH, GameraGPU, GamParams, GEOMETRY_ARRAYS
from oracle.oracle import Oracle, OracleParams

# oracle array name -> C-ABI geometry name
GEO_FROM_ORACLE = {"face": "face", "xfc": "xfc", "Tf": "Tf", "volume": "volume", "xyzcc": "xyzcc", "di": "di",
                   "dj": "dj", "dk": "dk", "edge": "edge", "Te": "Te", "Teb": "Teb"}


def make_oracle(problem: str, N, variant="strict", **kw):
    Nip, Njp, Nkp = N
    if problem == "ot":
        xyz = grids.uniform_corners(Nip, Njp, Nkp)
    elif problem == "bw":
        xyz = grids.warped_periodic_corners(Nip, Njp, Nkp)
    else:
        raise ValueError(problem)
    p = OracleParams(Nip, Njp, Nkp, do25D=(Nkp == 1), **kw)
    o = Oracle(p, xyz, variant)
    if problem == "ot":
        o.ic_orszag_tang()
    else:
        o.ic_blast_wave()
    st = o.init_finish()
    assert st == 0
    return o, xyz


def gpu_from_oracle(o: Oracle, precision=0, strict=False, lib_path=LIB_PATH, **kw) -> GameraGPU:
    p = o.p
    args = dict(gamma=p.gamma, CFL=p.CFL, pdmb=p.pdmb, Vd0=p.Vd0, cHogH=p.cHogH, cHogM=p.cHogM, dFloor=p.dFloor,
                pFloor=p.pFloor, tFin=p.tFin, dt0=p.dt0, limDT0=p.limDT0, rmeth=1 if p.up7 else 0,
                doLFMLim=p.doLFMLim, doMHD=p.doMHD, do25D=p.do25D, precision=precision, strict=strict)
    args.update(kw)
    g = GameraGPU(GamParams(p.Nip, p.Njp, p.Nkp, **args), lib_path=lib_path)
    g.set_geometry_arrays({n: o.array(GEO_FROM_ORACLE[n]) for n, _, _ in GEOMETRY_ARRAYS})
    sc = o.scalars()
    g.upload_state(o.array("Gas"), o.array("magFlux"), o.array("Bxyz"), o.array("oGas"), o.array("omagFlux"),
                   sc["time"], sc["otime"], sc["dt"], sc["ts"])
    return g


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
