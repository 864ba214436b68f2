"""Writes the golden fixtures of tests/golden (run once; needs mpmath).

gamutils_kat.json : the known-answer tests of the reference's
                    tests/gamera/testgamutils.pf:24-112 (CellP2C / CellC2P,
                    gamma = 5/3) with their tolerances, transcribed as data.
metric_kat.json   : tests/gamera/testmetric.pf: corner/face/cell coordinates of
                    the box with corners (1,1,1) and (2,3,4), as data.
erfc_exp.json     : erfc(x) and exp(x) at 40 significant digits (mpmath) on a
                    fixed set of points, the reference values for the
                    self-written FP64 erfc/exp.
"""
import json
import os

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    kat = {
        "gamma": "5/3",
        "prim": [0.1, 0.2, 0.3, 0.4, "2/3"],
        "con": [0.1, 0.02, 0.03, 0.04, 1.0145],
        "p2c_tol": [0.0, 1e-16, 1e-16, 1e-16, 2e-16],
        "c2p_tol": [0.0, 1e-16, 1e-16, 1e-16, 2e-16],
        "c2c_tol": [0.0, 2e-16, 2e-16, 2e-16, 4e-16],
        "p2p_tol": [0.0, 2e-16, 2e-16, 2e-16, 4e-16],
        "source": "tests/gamera/testgamutils.pf:24-112",
    }
    with open(os.path.join(HERE, "gamutils_kat.json"), "w") as f:
        json.dump(kat, f, indent=1)

    met = {
        "corners_lo": [1, 1, 1], "corners_hi": [2, 3, 4],
        "cell_center": [1.5, 2.0, 2.5],
        "face_center": {"I": [1.0, 2.0, 2.5], "J": [1.5, 1.0, 2.5], "K": [1.5, 2.0, 1.0]},
        "face_coords": {"I": [[1, 1, 1], [1, 3, 1], [1, 1, 4], [1, 3, 4]],
                        "J": [[1, 1, 1], [1, 1, 4], [2, 1, 1], [2, 1, 4]],
                        "K": [[1, 1, 1], [2, 1, 1], [1, 3, 1], [2, 3, 1]]},
        "edge_coords": {"I": [[1, 1, 1], [2, 1, 1]], "J": [[1, 1, 1], [1, 3, 1]], "K": [[1, 1, 1], [1, 1, 4]]},
        "source": "tests/gamera/testmetric.pf",
    }
    with open(os.path.join(HERE, "metric_kat.json"), "w") as f:
        json.dump(met, f, indent=1)

    mp.mp.dps = 50
    rng = np.random.default_rng(20261203)
    xs = np.concatenate([np.linspace(-6, 6, 49), rng.uniform(-6, 6, 200), rng.uniform(6, 26, 100),
                         [0.0, 1e-300, 1e-8, 0.5, 1.0, 2.0, 26.0]])
    es = np.concatenate([np.linspace(-700, 700, 57), rng.uniform(-40, 40, 200), [0.0, 1e-10, -1e-10]])
    data = {
        "erfc": [[float(x).hex(), mp.nstr(mp.erfc(mp.mpf(float(x))), 40)] for x in xs],
        "exp": [[float(x).hex(), mp.nstr(mp.exp(mp.mpf(float(x))), 40)] for x in es],
    }
    with open(os.path.join(HERE, "erfc_exp.json"), "w") as f:
        json.dump(data, f, indent=0)


if __name__ == "__main__":
    main()
