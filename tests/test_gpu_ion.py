"""The ionospheric inner boundary and its model hooks through the C ABI
(bc[0] = GAM_BC_ION, gam_set_ionosphere: IonInner with CellPlasmaBC, HackE =
IonEFix + WindEFix with DiffuseOuter + FixEFieldLFM, HackStep = PushIon +
NudgeSW; voltron/ICs/earthcmi.F90, apps/wind.F90) on the dipole in the
solar wind, against the oracle's restatement:

* strict build vs the oracle built with the same erfc/exp: initial state and
  1 + 9 steps identical bit for bit (State, oState, dt, t), with and without
  PushIon, and after the coupling fields are replaced between steps;
* product build within 1e-11 relative after 10 steps; FP32 form within
  1e-5 relative L2 of FP64 per conserved variable after 10 steps;
* the boundary needs its fields before the initial condition (GAM_ESTATE)
  and k-periodic boundaries (GAM_EINVAL for k-slabs).
"""
import numpy as np
import pytest

from mage_b200 import dipole, grids
from mage_b200.gamera import (BACKGROUND_ARRAYS, BC_HALO, BC_ION, BC_PERIODIC, BC_WIND, BC_ZEROGRAD, FP32,
                              GAM_EINVAL, GAM_ESTATE, GamError, GameraGPU, GamParams)
from oracle.oracle import Oracle, OracleParams
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

BCS = (BC_ION, BC_WIND, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)
WIND = dipole.wind_code_units()
SEED, AMP = 31337, 0.01
STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")
N = (16, 8, 8)
DTCPL = 5.0 / 63.8


def _fields(seed):
    rng = np.random.default_rng(seed)
    return (200.0 * rng.standard_normal((3, N[2] + 8, N[1] + 8, 5)),
            200.0 * rng.standard_normal((3, N[2] + 9, N[1] + 9, 6)))


def _pair(push, variant="gm", **kw):
    xyz = grids.spherical_corners(*N)
    o = Oracle(OracleParams(*N, doBackground=True, M0=dipole.M0, wind=WIND, bc=BCS), xyz, variant)
    E, Ee = _fields(7)
    o.set_ionosphere(E, Ee, dipole.M0, DTCPL, push, 2)
    o.ic_dipole_wind(AMP, SEED)
    assert o.init_finish() == 0
    g = GameraGPU(GamParams(*N, doBackground=1, bc=BCS, **kw))
    g.set_geometry(xyz)
    g.set_background({n: o.array(n) for n, _ in BACKGROUND_ARRAYS})
    g.set_ionosphere(E, Ee, dipole.M0, DTCPL, push, 2)
    g.init_dipole_wind(WIND, SEED, AMP)
    return o, g


@pytest.mark.parametrize("push", [True, False], ids=["push", "nopush"])
def test_ionosphere_strict_is_bit_exact(oracle_built, push):
    o, g = _pair(push, strict=True)
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), ("init", k, rel_err(s[k], o.array(k)))
    for nst in (1, 9):
        assert o.step(nst) == 0
        dt, t = g.step_gamera(nst)
        s = g.download_state()
        for k in STATE:
            assert np.array_equal(s[k], o.array(k)), (nst, k, rel_err(s[k], o.array(k)))
        sc = o.scalars()
        assert dt == sc["dt"] and t == sc["t"]
    # the coupler hands over new fields: both sides take them from the next step
    E, Ee = _fields(8)
    o.set_ionosphere(E, Ee, dipole.M0, DTCPL, push, 2)
    g.set_ionosphere(E, Ee, dipole.M0, DTCPL, push, 2)
    assert o.step(3) == 0
    g.step_gamera(3)
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), ("new fields", k, rel_err(s[k], o.array(k)))


def test_ionosphere_product_and_fp32(oracle_built):
    o, g = _pair(True, variant="strict")
    assert o.step(10) == 0
    g.step_gamera(10)
    s = g.download_state()
    for k in ("Gas", "magFlux"):
        assert rel_err(s[k], o.array(k)) <= 1e-11, (k, rel_err(s[k], o.array(k)))
    _, g32 = _pair(True, variant="strict", precision=FP32)
    g32.step_gamera(10)
    s32 = g32.download_state()
    ref = o.array("Gas")
    for v in range(5):
        err = np.linalg.norm(s32["Gas"][v] - ref[v]) / np.linalg.norm(ref[v])
        assert err <= 1e-5, (v, err)


def test_ionosphere_needs_its_fields():
    xyz = grids.spherical_corners(*N)
    g = GameraGPU(GamParams(*N, doBackground=1, bc=BCS))
    g.set_geometry(xyz)
    g.set_background_dipole(dipole.M0)
    with pytest.raises(GamError) as e:
        g.init_dipole_wind(WIND, SEED, AMP)
    assert e.value.args[0].startswith("GAM_ESTATE")
    with pytest.raises(GamError) as e:
        GameraGPU(GamParams(*N, doBackground=1, bc=BCS[:4] + (BC_HALO, BC_HALO)))
    assert e.value.args[0].startswith("GAM_EINVAL")
