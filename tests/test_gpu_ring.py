"""Ring averaging about the LFM axis on the GPU (bc[2] = bc[3] = GAM_BC_LFM,
gam_set_rings: the pole boundaries, RingGridFix, RingFlux, PoleE,
RingAverage, the deferred CalcDT) against the oracle's restatement, on a grid
spherical about the x axis (mage_b200.grids.lfm_corners):

* the metric with RingGridFix and the initial state equal the oracle's bit
  for bit;
* the strict build equals the oracle (built with the same erfc/exp) bit for
  bit after 1 and 10 steps of an off-axis blast wave: one ring of 8 chunks
  (PPM), 4 chunks with PLM, PCM without Fourier cleaning or loop cleaning,
  two Fourier modes removed, and the reference's two-ring default for 32
  cells around the axis;
* the magnetosphere on the LFM grid (ionospheric inner boundary with its
  hooks, solar wind, both poles with rings): bit for bit after 1 and 10
  steps with the ring branches of IonInner, WindBC, WindEFix and NudgeSW;
* the product build within 1e-11 and the FP32 form within 1e-5 relative L2
  of the oracle after 10 steps;
* the same magnetosphere cut 2 x 2 in i and j (each pole's rings on the
  tiles that hold it) equals the single grid bit for bit;
* the bounds-check build runs the ring configurations with no check firing.
"""
import numpy as np
import pytest

from mage_b200 import dipole, grids
from mage_b200.gamera import (BACKGROUND_ARRAYS, BC_ION, BC_LFM, BC_PERIODIC, BC_SPHIN, BC_WIND, BC_ZEROGRAD,
                              CHECK_LIB_PATH, FP32, LIB_PATH, RING_PCM, RING_PLM, GameraGPU, GamParams,
                              ring_defaults)
from mage_b200.tiling import Tiles, tile_box, tile_cut
from oracle.oracle import Oracle, OracleParams
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")
BW = dict(x0=6.0, y0=0.7, z0=0.0, rC=3.0, B0=0.3)
BCS = (BC_SPHIN, BC_ZEROGRAD, BC_LFM, BC_LFM, BC_PERIODIC, BC_PERIODIC)
GEO = ("face", "Tf", "volume", "dk", "di", "dj", "edge", "Te", "Teb")


def _blast(N, nch, recon=0, nft=1, clean=True, variant="gm", lib_path=LIB_PATH, **kw):
    xyz = grids.lfm_corners(*N, th0=0.01)
    o = Oracle(OracleParams(*N, bc=BCS, ringNch=tuple(nch), ringRecon=recon, ringNFT=nft, ringClean=clean), xyz,
               variant)
    o.ic_blast_wave(**BW)
    assert o.init_finish() == 0
    g = GameraGPU(GamParams(*N, bc=BCS, **kw), lib_path=lib_path)
    g.set_rings(nch, recon, nft, clean)
    g.set_geometry(xyz)
    g.init_blast_wave(**BW)
    return o, g


def _bitwise(o, g, tag):
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), (tag, k, rel_err(s[k], o.array(k)))
    sc = o.scalars()
    assert s["dt"] == sc["dt"] and s["time"] == sc["time"], tag


CASES = {
    "ppm8": ((16, 16, 16), (8,), 0, 1, True),
    "plm4": ((16, 16, 16), (4,), RING_PLM, 1, True),
    "pcm-noclean": ((16, 16, 16), (8,), RING_PCM, -1, False),
    "two-modes": ((16, 16, 16), (8,), 0, 2, True),
    "two-rings": ((16, 16, 32), None, 0, 1, True),
}


@pytest.mark.parametrize("case", list(CASES))
def test_rings_strict_is_bit_exact(oracle_built, case):
    N, nch, recon, nft, clean = CASES[case]
    if nch is None:
        nch = ring_defaults(N[2])
        assert nch == [8, 16]
    o, g = _blast(N, nch, recon, nft, clean, strict=True)
    geo = g.get_geometry_arrays()
    for n in GEO:
        assert np.array_equal(geo[n], o.array(n)), (case, n)
    _bitwise(o, g, (case, "init"))
    for nst in (1, 9):
        assert o.step(nst) == 0
        g.step_gamera(nst)
        _bitwise(o, g, (case, nst))


def test_rings_product_and_fp32(oracle_built):
    N = (16, 16, 16)
    o, g = _blast(N, (8,), variant="strict")
    assert o.step(10) == 0
    g.step_gamera(10)
    s = g.download_state()
    for k in ("Gas", "magFlux"):
        assert rel_err(s[k], o.array(k)) <= 1e-11, (k, rel_err(s[k], o.array(k)))
    _, g32 = _blast(N, (8,), variant="strict", precision=FP32)
    g32.step_gamera(10)
    s32 = g32.download_state()
    ref = o.array("Gas")
    for v in range(5):
        err = np.linalg.norm(s32["Gas"][v] - ref[v]) / np.linalg.norm(ref[v])
        assert err <= 1e-5, (v, err)


MBCS = (BC_ION, BC_WIND, BC_LFM, BC_LFM, BC_PERIODIC, BC_PERIODIC)
WIND = dipole.wind_code_units()
DTCPL = 5.0 / 63.8


def _fields(N, seed=7):
    rng = np.random.default_rng(seed)
    return (200.0 * rng.standard_normal((3, N[2] + 8, N[1] + 8, 5)),
            200.0 * rng.standard_normal((3, N[2] + 9, N[1] + 9, 6)))


def test_magnetosphere_rings_strict_is_bit_exact(oracle_built):
    N = (16, 8, 16)
    xyz = grids.lfm_corners(*N, th0=0.01)
    E, Ee = _fields(N)
    o = Oracle(OracleParams(*N, doBackground=True, M0=dipole.M0, wind=WIND, bc=MBCS, ringNch=(8,)), xyz, "gm")
    o.set_ionosphere(E, Ee, dipole.M0, DTCPL, True, 2)
    o.ic_dipole_wind(0.01, 31337)
    assert o.init_finish() == 0
    g = GameraGPU(GamParams(*N, doBackground=1, bc=MBCS, strict=True))
    g.set_rings([8])
    g.set_geometry(xyz)
    g.set_background({n: o.array(n) for n, _ in BACKGROUND_ARRAYS})
    g.set_ionosphere(E, Ee, dipole.M0, DTCPL, True, 2)
    g.init_dipole_wind(WIND, 31337, 0.01)
    _bitwise(o, g, "init")
    for nst in (1, 9):
        assert o.step(nst) == 0
        g.step_gamera(nst)
        _bitwise(o, g, nst)


def test_magnetosphere_rings_tiles_equal_single_grid():
    N, dims = (32, 16, 16), (2, 2, 1)
    xyz = grids.lfm_corners(*N, th0=0.01)
    E, Ee = _fields(N)
    one = GameraGPU(GamParams(*N, doBackground=1, bc=MBCS, strict=True))
    one.set_rings([8])
    one.set_geometry(xyz)
    one.set_background_dipole(dipole.M0)
    one.set_ionosphere(E, Ee, dipole.M0, DTCPL, True, 2)
    one.init_dipole_wind(WIND, 31337, 0.01)
    one.step_gamera(2)
    s0 = one.download_state()

    def setup(g, t):
        g.set_background_dipole(dipole.M0)
        if t.bc[1] == BC_WIND:
            g.set_wind(WIND)
        if t.bc[0] == BC_ION:
            g.set_ionosphere(tile_cut(E, 2, N[1], dims[1], t.t[1]), tile_cut(Ee, 2, N[1], dims[1], t.t[1]),
                             dipole.M0, DTCPL, True, 2)
        else:
            g.set_ionosphere(None, None, dipole.M0, DTCPL, True, 2)
        st = {k: tile_box(s0[k], N, dims, t.t) for k in STATE}
        g.upload_state(st["Gas"], st["magFlux"], st["Bxyz"], st["oGas"], st["omagFlux"], s0["time"], s0["otime"],
                       s0["dt"], s0["ts"])

    tl = Tiles(N, xyz, dims, strict=True, bc=MBCS, problem=setup, params={"doBackground": 1},
               rings={"Nch": [8]})
    for n in (1, 6):
        assert one.step_gamera(n) == tl.step(n)
        ref = one.download_state()
        for t, g in zip(tl.tiles, tl.apps):
            s = g.download_state()
            for k in ("Gas", "Bxyz", "oGas"):
                assert np.array_equal(s[k], tile_box(ref[k], N, dims, t.t)), (n, t.t, k)
            for k in ("magFlux", "omagFlux"):
                a, b = s[k], tile_box(ref[k], N, dims, t.t)
                assert np.array_equal(a[0][:-1, :-1, :], b[0][:-1, :-1, :]), (n, t.t, k, "I")
                assert np.array_equal(a[1][:-1, :, :-1], b[1][:-1, :, :-1]), (n, t.t, k, "J")
                assert np.array_equal(a[2][:, :-1, :-1], b[2][:, :-1, :-1]), (n, t.t, k, "K")


def test_rings_checked_build():
    N = (16, 16, 16)
    xyz = grids.lfm_corners(*N, th0=0.01)
    g = GameraGPU(GamParams(*N, bc=BCS, strict=True), lib_path=CHECK_LIB_PATH)
    g.set_rings([4], RING_PLM)
    g.set_geometry(xyz)
    g.init_blast_wave(**BW)
    g.step_gamera(4)
    assert g.bounds_status()["fired"] == 0
    E, Ee = _fields(N)
    m = GameraGPU(GamParams(*N, doBackground=1, bc=MBCS), lib_path=CHECK_LIB_PATH)
    m.set_rings([8])
    m.set_geometry(xyz)
    m.set_background_dipole(dipole.M0)
    m.set_ionosphere(E, Ee, dipole.M0, DTCPL, True, 2)
    m.init_dipole_wind(WIND, 31337, 0.01)
    m.step_gamera(4)
    assert m.bounds_status()["fired"] == 0
