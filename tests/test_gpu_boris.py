"""Boris correction (physics/doBoris with the speed of light Ca, init.F90:417-423)
through the C ABI: the Boris-limited Alfven speed of the electric field
(fields.F90:211-213), MagKinFlux (stress.F90:560-564), CellDT
(gridutils.F90:91-93) and Con2Fast (gamutils.F90:356-358), the Boris hogs of
the magnetic fluxes (stress.F90:335-349), the nuclear option of the gas fluxes
(stress.F90:399-417) and CellBoris in the update (mhdgroup.F90:334-382).

* strict build: Orszag-Tang with Ca = 0.5 (below the vortex speed, so the
  nuclear option fires) and the dipole in the wind with Ca = 10 (background
  field in CellBoris, Boris Con2Fast in the wind): initial state and N steps
  identical, bit for bit, to the oracle built with the same erfc/exp;
* product FP64 build: <= 1e-12 relative to the oracle after 20 steps; FP32
  form vs FP64: relative L2 per conserved variable, bound in the test;
* the adjoint stages, which differentiate the step without Boris, refuse it.
"""
import ctypes as C

import numpy as np
import pytest

from mage_b200 import dipole, grids
from mage_b200.gamera import (BACKGROUND_ARRAYS, BC_PERIODIC, BC_SPHIN, BC_WIND, BC_ZEROGRAD, FP32, GameraGPU,
                              GamParams, load_library)
from oracle.oracle import Oracle, OracleParams
from tests.helpers import gpu_from_oracle, make_oracle, rel_err

pytestmark = pytest.mark.gpu

STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")
N_OT = (32, 32, 4)
CA_OT = 0.5


def _ot(variant="gm", **kw):
    """Oracle start and metric handed to the GPU through the C ABI."""
    o, _ = make_oracle("ot", N_OT, variant=variant, doBoris=True, Ca=CA_OT)
    return o, gpu_from_oracle(o, doBoris=True, Ca=CA_OT, **kw)


def _same(o, g, tag):
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), (tag, k, rel_err(s[k], o.array(k)))
    return s


def test_boris_orszag_tang_strict_is_bit_exact(oracle_built):
    o, g = _ot(strict=True)
    _same(o, g, "init")
    for nst in (1, 9):
        assert o.step(nst) == 0
        dt, _ = g.step_gamera(nst)
        _same(o, g, nst)
        assert dt == o.scalars()["dt"]


def test_boris_dipole_strict_is_bit_exact(oracle_built):
    N = (16, 8, 8)
    bcs = (BC_SPHIN, BC_WIND, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)
    w = dipole.wind_code_units()
    xyz = grids.spherical_corners(*N)
    o = Oracle(OracleParams(*N, doBackground=True, M0=dipole.M0, wind=w, bc=bcs, doBoris=True, Ca=10.0), xyz, "gm")
    o.ic_dipole_wind(0.01, 31337)
    assert o.init_finish() == 0
    g = GameraGPU(GamParams(*N, doBackground=1, bc=bcs, strict=True, doBoris=True, Ca=10.0))
    g.set_geometry(xyz)
    g.set_background({n: o.array(n) for n, _ in BACKGROUND_ARRAYS})
    g.init_dipole_wind(w, 31337, 0.01)
    _same(o, g, "init")
    for nst in (1, 9):
        assert o.step(nst) == 0
        dt, _ = g.step_gamera(nst)
        _same(o, g, nst)
        assert dt == o.scalars()["dt"]


def test_boris_product_and_fp32(oracle_built):
    o, g = _ot(variant="strict")
    assert o.step(20) == 0
    g.step_gamera(20)
    s = g.download_state()
    for k in ("Gas", "magFlux", "Bxyz"):
        assert rel_err(s[k], o.array(k)) <= 1e-12, (k, rel_err(s[k], o.array(k)))
    # FP32 form on the same start
    _, g32 = _ot(variant="strict", precision=FP32)
    g32.step_gamera(20)
    s32 = g32.download_state()
    a, b = s32["Gas"][:, 4:8, 4:36, 4:36], s["Gas"][:, 4:8, 4:36, 4:36]
    # density, momentum (as a vector: the 2.5-D vortex has no z momentum) and energy
    parts = [a[0:1] - b[0:1], a[1:4] - b[1:4], a[4:5] - b[4:5]], [b[0:1], b[1:4], b[4:5]]
    errs = [float(np.linalg.norm(d) / np.linalg.norm(r)) for d, r in zip(*parts)]
    print("FP32 vs FP64 relative L2 (rho, momentum, energy):", errs)
    assert max(errs) <= 1e-5, errs


def test_adjoint_stages_refuse_boris():
    L = load_library()
    p = GamParams(16, 16, 16, doBoris=True, Ca=1.0).to_c()
    dummy = C.c_void_p(1)
    rc = L.gam_flux_forward(C.byref(p), 0, *([dummy] * 8), None, None, dummy, dummy, None)
    assert rc == 1  # GAM_EINVAL
