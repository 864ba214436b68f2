"""The bounds-check build (libgamgpu_check.so, -DGAM_BOUNDS_CHECK) on small
grids: every kernel checks the box indices its stencils touch before any load,
and the device arrays start as NaN canaries instead of zeros.

* strict kernels of the checked build equal the oracle bit for bit (so no
  canary, i.e. no read of memory nothing wrote, reaches a result) and no
  check fires, over the configurations the step supports: curvilinear blast
  wave (with AB3, with Boris), 2.5-D Orszag-Tang, the dipole in the wind, the
  inflow / outflow boundaries, FP32, two emulated k-slabs and 2 x 2 x 2
  emulated tiles;
* the reporting path: a limit below the box size (GAM_BOUNDS_LIMIT, read at
  handle creation) makes in-bounds indices fail the check; the step returns
  GAM_EBOUNDS with the kernel recorded and no memory outside the box is
  touched (a failed check skips the access).
"""
import os

import numpy as np
import pytest

from mage_b200 import dipole, grids
from mage_b200.gamera import (BACKGROUND_ARRAYS, BC_INFLOW, BC_PERIODIC, BC_SPHIN, BC_WIND, BC_ZEROGRAD,
                              CHECK_LIB_PATH, FP32, GAM_EBOUNDS, GamError, GameraGPU, GamParams)
from oracle.oracle import Oracle, OracleParams
from tests.helpers import gpu_from_oracle, make_oracle, rel_err

pytestmark = pytest.mark.gpu

STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")


def _bitwise(o, g, tag):
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), (tag, k, rel_err(s[k], o.array(k)))
    st = g.bounds_status()
    assert st["fired"] == 0, (tag, st)


@pytest.mark.parametrize("prob,N,kw", [("bw", (16, 16, 16), {}), ("bw", (16, 16, 16), {"doAB3": True}),
                                      ("bw", (16, 16, 16), {"doBoris": True, "Ca": 0.5}), ("ot", (32, 32, 1), {})],
                         ids=["bw", "bw-ab3", "bw-boris", "ot-2.5d"])
def test_checked_build_periodic(oracle_built, prob, N, kw):
    o, _ = make_oracle(prob, N, variant="gm", **kw)
    g = gpu_from_oracle(o, strict=True, lib_path=CHECK_LIB_PATH, **kw)
    assert g.bounds_status()["fired"] == 0
    assert o.step(6) == 0
    g.step_gamera(6)
    _bitwise(o, g, (prob, kw))


def test_checked_build_dipole_and_inflow(oracle_built):
    N = (16, 8, 8)
    bcs = (BC_SPHIN, BC_WIND, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)
    w = dipole.wind_code_units()
    xyz = grids.spherical_corners(*N)
    o = Oracle(OracleParams(*N, doBackground=True, M0=dipole.M0, wind=w, bc=bcs), xyz, "gm")
    o.ic_dipole_wind(0.01, 31337)
    assert o.init_finish() == 0
    g = GameraGPU(GamParams(*N, doBackground=1, bc=bcs, strict=True), lib_path=CHECK_LIB_PATH)
    g.set_geometry(xyz)
    g.set_background({n: o.array(n) for n, _ in BACKGROUND_ARRAYS})
    g.init_dipole_wind(w, 31337, 0.01)
    assert o.step(6) == 0
    g.step_gamera(6)
    _bitwise(o, g, "dipole")

    N = (16, 12, 12)
    bcs = (BC_INFLOW, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC)
    inflow = (1.0, 0.1, 0.5, 0.0, 0.0, 0.5 ** 0.5, 0.5 ** 0.5, 0.3)
    xyz = grids.warped_periodic_corners(*N)
    o = Oracle(OracleParams(*N, bc=bcs, inflow=inflow), xyz, "gm")
    o.ic_blast_wave()
    assert o.init_finish() == 0
    g = GameraGPU(GamParams(*N, bc=bcs, strict=True), lib_path=CHECK_LIB_PATH)
    g.set_geometry(xyz)
    g.set_inflow(inflow)
    g.init_blast_wave()
    assert o.step(6) == 0
    g.step_gamera(6)
    _bitwise(o, g, "inflow")


def test_checked_build_fp32_and_slabs(oracle_built):
    from mage_b200.tiling import Slabs
    o, _ = make_oracle("bw", (16, 16, 16), variant="strict")
    g = gpu_from_oracle(o, precision=FP32, lib_path=CHECK_LIB_PATH)
    assert o.step(6) == 0
    g.step_gamera(6)
    s = g.download_state()
    assert g.bounds_status()["fired"] == 0
    assert rel_err(s["Gas"], o.array("Gas")) <= 1e-5
    N = (16, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    sl = Slabs(N, xyz, 2, strict=True, lib_path=CHECK_LIB_PATH)
    sl.step(4)
    for a in sl.apps:
        assert a.bounds_status()["fired"] == 0


def test_checked_build_tiles():
    """Tiles along i, j and k: the halo kernels of every direction and side
    stay inside the box, and the tiles equal the checked single grid."""
    from mage_b200.tiling import Tiles, tile_box
    N = (32, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    one = GameraGPU(GamParams(*N, strict=True), lib_path=CHECK_LIB_PATH)
    one.set_geometry(xyz)
    one.init_blast_wave()
    tl = Tiles(N, xyz, (2, 2, 2), strict=True, lib_path=CHECK_LIB_PATH)
    assert one.step_gamera(3) == tl.step(3)
    ref = one.download_state()
    assert one.bounds_status()["fired"] == 0
    for t, a in zip(tl.tiles, tl.apps):
        assert a.bounds_status()["fired"] == 0
        assert np.array_equal(a.download_state()["Gas"], tile_box(ref["Gas"], N, tl.dims, t.t)), t.t


def test_bounds_report_path():
    """GAM_BOUNDS_LIMIT = 1000 elements: every index at or above it fails the
    check (all of them in bounds of the real box), so the first kernels with
    checks (the initial boundary fill and CalcDT) report."""
    os.environ["GAM_BOUNDS_LIMIT"] = "1000"
    try:
        N = (16, 16, 16)
        g = GameraGPU(GamParams(*N), lib_path=CHECK_LIB_PATH)
    finally:
        del os.environ["GAM_BOUNDS_LIMIT"]
    g.set_geometry(grids.warped_periodic_corners(*N))
    with pytest.raises(GamError) as e:  # the first fill of the boundaries and CalcDT already report
        g.init_blast_wave()
        g.step_gamera(1)
    assert e.value.code == GAM_EBOUNDS
    st = g.bounds_status()
    assert st["fired"] == 1 and 1 <= st["kernel"] <= 16 and st["index"] >= 1000, st
