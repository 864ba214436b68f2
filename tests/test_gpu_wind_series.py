"""Solar-wind time series on the outer-I boundary (gam_set_wind_series;
WindBC with RefreshWind / GetWindAt / wgtWind / InterpWind,
apps/wind.F90:116-203, 206-391, 766-868) for the dipole in the wind.

The weights of a series are evaluated on the device with CUDA's acos and exp,
the CPU restatement's with libm's, so the comparisons carry a tolerance
instead of bit equality:
* a series whose rows all hold the constant wind reproduces the constant-wind
  run (host-side libm weights) to <= 1e-12 relative after 10 steps;
* a varying, tilted-front series (rows every 0.5 time units, lag times up to
  ~7.5 across the grid, so ghost cells and faces see different rows): the
  strict build agrees with the oracle to <= 1e-12, the product build to
  <= 1e-11;
* a series faster than the Boris speed is refused, like readWind does.
"""
import numpy as np
import pytest

from mage_b200 import dipole, grids
from mage_b200.gamera import (BACKGROUND_ARRAYS, BC_PERIODIC, BC_SPHIN, BC_WIND, BC_ZEROGRAD, GAM_EINVAL, GamError,
                              GameraGPU, GamParams)
from oracle.oracle import Oracle, OracleParams
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

N = (16, 8, 8)
BCS = (BC_SPHIN, BC_WIND, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)
W = dipole.wind_code_units()


def _const_series():
    n = 21
    t = np.linspace(-100.0, 100.0, n)
    return dict(t=t, rho=np.full(n, W[0]), P=np.full(n, W[1]), V=np.tile(W[2:5], (n, 1)), B=np.tile(W[5:8], (n, 1)),
                Bx0=W[5])


def _varying_series():
    t = np.arange(-10.0, 10.01, 0.5)
    n = t.size
    V = np.tile(W[2:5], (n, 1)) * (1.0 + 0.05 * np.cos(t))[:, None]
    V[:, 1] = 0.3 * np.sin(t)
    B = np.tile(W[5:8], (n, 1))
    B[:, 1] = 0.4 * np.cos(0.7 * t)
    B[:, 2] = W[7] * (1.0 + 0.2 * np.sin(t))
    return dict(t=t, rho=W[0] * (1.0 + 0.1 * np.sin(t)), P=W[1] * (1.0 + 0.1 * np.cos(t)), V=V, B=B, Bx0=0.1,
                ByC=0.2, BzC=-0.1)


def _oracle(series, variant):
    xyz = grids.spherical_corners(*N)
    o = Oracle(OracleParams(*N, doBackground=True, M0=dipole.M0, wind=W, bc=BCS), xyz, variant)
    o.ic_dipole_wind(0.01, 31337)
    if series is not None:
        o.set_wind_series(**series)
    assert o.init_finish() == 0
    return o


def _gpu(o, series, **kw):
    g = GameraGPU(GamParams(*N, doBackground=1, bc=BCS, **kw))
    g.set_geometry(grids.spherical_corners(*N))
    g.set_background({n: o.array(n) for n, _ in BACKGROUND_ARRAYS})
    g.init_dipole_wind(W, 31337, 0.01)
    if series is not None:
        g.set_wind_series(**series)
        # the first fill used the constant wind; hand over the oracle's start
        sc = o.scalars()
        g.upload_state(o.array("Gas"), o.array("magFlux"), o.array("Bxyz"), o.array("oGas"), o.array("omagFlux"),
                       sc["time"], sc["otime"], sc["dt"], sc["ts"])
    return g


def test_constant_rows_reproduce_the_constant_wind(oracle_built):
    o = _oracle(None, "gm")
    a = _gpu(o, None, strict=True)
    b = _gpu(o, _const_series(), strict=True)
    a.step_gamera(10)
    b.step_gamera(10)
    sa, sb = a.download_state(), b.download_state()
    for k in ("Gas", "magFlux", "Bxyz"):
        assert rel_err(sb[k], sa[k]) <= 1e-12, (k, rel_err(sb[k], sa[k]))


@pytest.mark.parametrize("strict,tol", [(True, 1e-12), (False, 1e-11)], ids=["strict", "product"])
def test_varying_series_against_oracle(oracle_built, strict, tol):
    ser = _varying_series()
    o = _oracle(ser, "gm" if strict else "strict")
    g = _gpu(o, ser, strict=strict)
    assert o.step(10) == 0
    g.step_gamera(10)
    s = g.download_state()
    for k in ("Gas", "magFlux", "Bxyz"):
        assert rel_err(s[k], o.array(k)) <= tol, (k, rel_err(s[k], o.array(k)))
    # the series changed the solution against the constant wind
    c = _oracle(None, "strict")
    assert c.step(10) == 0
    assert rel_err(o.array("Gas"), c.array("Gas")) > 1e-6


def test_series_faster_than_boris_speed_is_refused():
    g = GameraGPU(GamParams(*N, doBackground=1, bc=BCS, doBoris=True, Ca=3.0))
    with pytest.raises(GamError) as e:
        g.set_wind_series(**_const_series())  # |V| = 4 >= Ca
    assert e.value.code == GAM_EINVAL
