"""The AB3 predictor (sim/doAB3, init.F90:377; Predictor and ExtrapAB3,
mhdgroup.F90:444-517, 721-731) through the C ABI.

* strict build: State, oState and ooState (face fluxes and time) identical,
  bit for bit, to the oracle built with the same erfc/exp after 1 and 10
  steps of a curvilinear blast wave and of 2.5-D Orszag-Tang;
* gam_set_oostate: a run continued from the oracle's State, oState and
  ooState after 5 steps stays bit-exact; gam_upload_state alone sets ooState =
  oState at otime - dt (the restart fallback, gioH5.F90:797-802);
* product FP64 build: <= 1e-12 relative to the oracle after 20 steps.
"""
import numpy as np
import pytest

from tests.helpers import gpu_from_oracle, make_oracle, rel_err

pytestmark = pytest.mark.gpu

STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")


def _check(o, g, tag):
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), (tag, k, rel_err(s[k], o.array(k)))
    oo = g.get_oostate()
    assert np.array_equal(oo["oomagFlux"], o.array("oomagFlux")), (tag, rel_err(oo["oomagFlux"], o.array("oomagFlux")))
    sc = o.scalars()
    assert oo["ootime"] == sc["ootime"] and s["otime"] == sc["otime"], (tag, oo["ootime"], sc["ootime"])


@pytest.mark.parametrize("prob,N", [("bw", (16, 16, 16)), ("ot", (32, 32, 1))], ids=["bw16", "ot32-2.5d"])
def test_ab3_strict_is_bit_exact(oracle_built, prob, N):
    o, _ = make_oracle(prob, N, variant="gm", doAB3=True)
    g = gpu_from_oracle(o, strict=True, doAB3=True)
    _check(o, g, "init")
    for nst in (1, 9):
        assert o.step(nst) == 0
        dt, _ = g.step_gamera(nst)
        _check(o, g, nst)
        assert dt == o.scalars()["dt"]


def test_ab3_oostate_upload(oracle_built):
    o, _ = make_oracle("bw", (16, 16, 16), variant="gm", doAB3=True)
    assert o.step(5) == 0
    g = gpu_from_oracle(o, strict=True, doAB3=True)
    sc = o.scalars()
    oo = g.get_oostate()  # the fallback: ooState = oState one dt earlier
    assert np.array_equal(oo["oomagFlux"], o.array("omagFlux")) and oo["ootime"] == sc["otime"] - sc["dt"]
    g.set_oostate(o.array("oomagFlux"), sc["ootime"])
    _check(o, g, "upload")
    assert o.step(5) == 0
    g.step_gamera(5)
    _check(o, g, "continued")


def test_ab3_product_build(oracle_built):
    o, _ = make_oracle("bw", (32, 32, 32), variant="strict", doAB3=True)
    g = gpu_from_oracle(o, doAB3=True)
    assert o.step(20) == 0
    g.step_gamera(20)
    s = g.download_state()
    for k in ("Gas", "magFlux", "Bxyz"):
        assert rel_err(s[k], o.array(k)) <= 1e-12, (k, rel_err(s[k], o.array(k)))
