"""Dipole in the solar wind on a spherical grid: background field (AddB0),
inner-sphere, solar-wind and zero-gradient boundaries, through the C ABI.

* strict build with the oracle's background arrays uploaded
  (gam_set_background, as a Fortran driver would hand over Grid%fcB0 ...):
  initial state and N steps identical, bit for bit, to the oracle built with
  the same erfc/exp;
* background field computed on the GPU (gam_set_background_dipole) vs the
  oracle's AddB0: <= 1e-13 relative; the two differ only through pow();
* FP32 form vs FP64 on the same start: relative L2 error per conserved
  variable, bound stated in the test.
"""
import numpy as np
import pytest

from mage_b200 import dipole, grids
from mage_b200.gamera import (BC_PERIODIC, BC_SPHIN, BC_WIND, BC_ZEROGRAD, FP32, GamError, GameraGPU, GamParams,
                              GEOMETRY_ARRAYS, BACKGROUND_ARRAYS, GAM_ESTATE, GAM_EINVAL)
from oracle.oracle import Oracle, OracleParams
from tests.helpers import GEO_FROM_ORACLE, rel_err

pytestmark = pytest.mark.gpu

STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")
BCS = (BC_SPHIN, BC_WIND, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)
WIND = dipole.wind_code_units()
SEED, AMP = 31337, 0.01


def _oracle(N, variant="gm"):
    xyz = grids.spherical_corners(*N)
    p = OracleParams(*N, doBackground=True, M0=dipole.M0, wind=WIND, bc=BCS)
    o = Oracle(p, xyz, variant)
    o.ic_dipole_wind(AMP, SEED)
    assert o.init_finish() == 0
    return o, xyz


def _gpu(o, xyz, **kw):
    p = o.p
    g = GameraGPU(GamParams(p.Nip, p.Njp, p.Nkp, gamma=p.gamma, CFL=p.CFL, doBackground=1, bc=BCS, **kw))
    g.set_geometry(xyz)
    return g


def test_dipole_wind_strict_is_bit_exact(oracle_built):
    o, xyz = _oracle((16, 8, 8))
    g = _gpu(o, xyz, strict=True)
    geo = g.get_geometry_arrays()
    for n, _, _ in GEOMETRY_ARRAYS:
        assert np.array_equal(geo[n], o.array(GEO_FROM_ORACLE[n])), n
    g.set_background({n: o.array(n) for n, _ in BACKGROUND_ARRAYS})
    g.init_dipole_wind(WIND, SEED, AMP)
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), ("init", k, rel_err(s[k], o.array(k)))
    assert s["dt"] == o.scalars()["dt"]
    for nst in (1, 9):
        assert o.step(nst) == 0
        dt, t = g.step_gamera(nst)
        s = g.download_state()
        for k in STATE:
            assert np.array_equal(s[k], o.array(k)), (nst, k, rel_err(s[k], o.array(k)))
        sc = o.scalars()
        assert dt == sc["dt"] and t == sc["t"] and s["ts"] == sc["ts"]
    # DivB with the background fluxes (gridutils.F90:717-770): same terms, another summation order
    assert abs(g.divb() - o.divb()) <= 1e-12 * o.divb()


def test_dipole_background_on_gpu(oracle_built):
    o, xyz = _oracle((16, 8, 8), variant="strict")
    g = _gpu(o, xyz)
    g.set_background_dipole(dipole.M0)
    bg = g.get_background()
    for n, _ in BACKGROUND_ARRAYS:
        ref = o.array(n)
        if n == "dpB0":
            # div of the dipole's Maxwell stress: zero analytically, round-off
            # of face stresses ~B^2 A; compare on that scale
            scale = np.abs(o.array("B0")).max() ** 2
            assert np.abs(bg[n] - ref).max() <= 1e-12 * scale, n
        else:
            assert rel_err(bg[n], ref) <= 1e-13, (n, rel_err(bg[n], ref))
    # stepping on the GPU background stays within round-off of the oracle
    g.init_dipole_wind(WIND, SEED, AMP)
    assert o.step(10) == 0
    g.step_gamera(10)
    s = g.download_state(old=False)
    for k in ("Gas", "magFlux", "Bxyz"):
        assert rel_err(s[k], o.array(k)) <= 1e-11, (k, rel_err(s[k], o.array(k)))


def test_dipole_fp32_form(oracle_built):
    o, xyz = _oracle((16, 8, 8), variant="strict")
    ref = o.array("Gas")
    a = _gpu(o, xyz)
    b = _gpu(o, xyz, precision=FP32)
    for g in (a, b):
        g.set_background({n: o.array(n) for n, _ in BACKGROUND_ARRAYS})
        g.init_dipole_wind(WIND, SEED, AMP)
    a.step_gamera(20)
    b.step_gamera(20)
    A = a.download_state(old=False)["Gas"][:, 4:-4, 4:-4, 4:-4]
    B = b.download_state(old=False)["Gas"][:, 4:-4, 4:-4, 4:-4]
    assert ref.shape[0] == 5
    for v in range(5):
        if np.abs(A[v]).max() > 1e-8:
            err = np.linalg.norm(B[v] - A[v]) / np.linalg.norm(A[v])
            assert err <= 1e-4, (v, err)


def test_wind_and_background_required():
    N = (16, 8, 8)
    g = GameraGPU(GamParams(*N, doBackground=1, bc=BCS))
    xyz = grids.spherical_corners(*N)
    g.set_geometry(xyz)
    with pytest.raises(GamError) as e:
        g.init_dipole_wind(WIND)
    assert e.value.code == GAM_ESTATE  # background first
    with pytest.raises(GamError) as e:
        GameraGPU(GamParams(*N, bc=(BC_PERIODIC, BC_PERIODIC, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)))
    assert e.value.code == GAM_EINVAL  # zero-gradient J with periodic I
    with pytest.raises(GamError) as e:
        GameraGPU(GamParams(*N, bc=(BC_WIND, BC_SPHIN, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC)))
    assert e.value.code == GAM_EINVAL  # wind is an outer-I kind
