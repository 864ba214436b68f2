"""Decks in the reference's XML format (mage_b200.deck): keys, defaults and
case rules of initModel (src/gamera/init.F90:312-484), SetFloors
(gamutils.F90:387-405) and Set_Val (src/base/io_xml_input.F90), no GPU work."""
import os

import numpy as np
import pytest

from mage_b200 import deck, grids
from mage_b200.gamera import RECON_8CENT

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "decks")


def test_defaults_of_init_model():
    d = deck.Deck(os.path.join(HERE, "ot2d_gpu.xml"))
    p = deck.params(d)
    assert (p.Nip, p.Njp, p.Nkp) == (32, 32, 1) and p.do25D  # one k layer: the 2.5-D step
    assert p.pdmb == 0.75 and p.CFL == min(0.5 / 1.25, 0.3) and p.Vd0 == 0.5
    assert p.gamma == 5.0 / 3.0 and p.cHogH == 0.25 and p.cHogM == 0.25
    assert p.dFloor == 1e-12 and p.pFloor == 1e-12 and p.limDT0 == 1e-3 and p.tFin == 0.05
    assert p.rmeth == RECON_8CENT and p.doLFMLim and p.doMHD and not p.doBoris and not p.doAB3
    assert p.fixedTimestep < 0


def test_every_key_kind_and_case():
    d = deck.Deck(os.path.join(HERE, "blast_gpu.xml"))
    p = deck.params(d)
    assert p.pdmb == 1.0 and p.CFL == 0.25 and p.Vd0 == 0.45 and p.doAB3
    assert p.dFloor == 1e-10 and p.pFloor == 1e-9  # floors/ read after sim/, Fortran 'd' exponent
    assert p.gamma == 1.4 and p.cHogH == 0.0 and p.cHogM == 0.0  # doHogs = F
    assert p.doBoris and p.Ca == 3.0 and p.limDT0 == 1e-4 and p.doMHD and not p.do25D
    bw = deck.blast_wave_args(d)
    assert bw == {"x0": 0.5, "y0": 0.5, "z0": 0.5, "D0": 1.0, "P0": 0.1, "pRat": 50.0, "dRat": 1.0, "rC": 0.1,
                  "B0": 0.5}
    assert np.array_equal(deck.corners(d), grids.uniform_corners(16, 16, 16))


@pytest.mark.parametrize("key", ["physics/doResistive", "multifluid/doMF", "grid/doSph", "restart/doRes"])
def test_unsupported_parts_are_refused(key):
    sec, k = key.split("/")
    text = (f'<Kaiju><Gamera><idir N="16"/><jdir N="16"/><kdir N="16"/><{sec} {k}="T"/></Gamera></Kaiju>')
    with pytest.raises(ValueError):
        deck.params(deck.Deck(text))


def test_fortran_logicals():
    for s, v in (("T", True), (".true.", True), ("t", True), ("F", False), (".FALSE.", False)):
        assert deck._bool(s) == v
    with pytest.raises(ValueError):
        deck._bool("yes")
