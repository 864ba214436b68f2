"""Decks in the reference's XML format run on the GPU (mage_b200.deck,
mage_b200.run): the 2.5-D Orszag-Tang deck runs to its tFin and lands on it,
keeps the vortex's mirror symmetry and div B at round-off, and logs one JSON
line per interval with the console block's fields; the blast-wave deck with
Boris and AB3 steps through the same path."""
import json
import os

import numpy as np
import pytest

from mage_b200 import deck
from mage_b200.run import run

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "decks")


def test_ot_deck_runs_to_tfin():
    lines = []
    last = run(os.path.join(HERE, "ot2d_gpu.xml"), every=5, emit=lines.append)
    recs = [json.loads(x) for x in lines]
    assert recs[-1] == last and last["status"] == "ok"
    assert abs(last["t"] - 0.05) <= 1e-12 and all(r["kZCs"] > 0 for r in recs)
    assert {"ts", "t", "dt", "dt/dt0", "kZCs", "divB", "totals"} <= set(last)
    assert last["divB"] <= 1e-10
    g, _ = deck.load(os.path.join(HERE, "ot2d_gpu.xml"))
    g.step_gamera(last["ts"])
    G = g.download_state(old=False)["Gas"][:, 4, 4:36, 4:36]
    F = G[:, ::-1, ::-1].copy()
    F[1:3] *= -1.0
    assert float(np.abs(G - F).max()) <= 1e-11 * float(np.abs(G).max())  # testCases.pf:198-216 bound


def test_blast_deck_with_boris_and_ab3():
    last = run(os.path.join(HERE, "blast_gpu.xml"), steps=6, every=3, emit=lambda s: None)
    assert last["status"] == "ok" and last["ts"] == 6
