"""The oracle's ionospheric inner boundary and its hooks (IonInner with
CellPlasmaBC, IonEFix + FixEFieldLFM, PushIon; voltron/ICs/earthcmi.F90) on
a small dipole-in-the-wind grid, against properties the reference code fixes
and an independent numpy evaluation of the E x B velocity:

* every ghost cell of the inner side carries the density and pressure of its
  mirror cell is+n-1 (k wrapped into the active range) and the velocity
  V = (E x B/|B|^2)_perp + min(Vr, 0) r^ of the coupling shell 5-n in the
  dipole field at the ghost cell's centre; every ghost-layer face has zero
  flux;
* PushIon with dtCpl far below dt moves the first shell's velocity onto the
  perpendicular E x B velocity of shell 5 (the push factor clips at 1);
* NudgeSW with dtSW0 far below dt puts the wind's velocity, density and
  pressure into every last active cell the wind reaches (weight > TINY);
* the step keeps div B at round-off and mass finite.
"""
import numpy as np
import pytest

from mage_b200 import dipole, grids
from oracle.oracle import Oracle, OracleParams

N = (12, 8, 8)
BCS = (7, 4, 2, 2, 0, 0)
G = 4


def _fields(seed):
    rng = np.random.default_rng(seed)
    inE = 200.0 * rng.standard_normal((3, N[2] + 8, N[1] + 8, 5))
    inEe = 200.0 * rng.standard_normal((3, N[2] + 9, N[1] + 9, 6))
    return inE, inEe


def _oracle(dtCpl=5.0 / 63.8, push=True, seed=5, dtSW0=60.0 / 63.8):
    xyz = grids.spherical_corners(*N)
    o = Oracle(OracleParams(*N, doBackground=True, M0=dipole.M0, wind=dipole.wind_code_units(), bc=BCS), xyz, "strict")
    inE, inEe = _fields(seed)
    o.set_ionosphere(inE, inEe, dipole.M0, dtCpl, push, 1, dtSW0)
    o.ic_dipole_wind(0.01, 31337)
    assert o.init_finish() == 0
    return o, inE


def _exb(xc, E, M0):
    """E x B / |B|^2 in the dipole of moment (0, 0, M0) at xc, and r^."""
    r = np.sqrt((xc ** 2).sum(axis=0))
    m = np.zeros_like(xc)
    m[2] = M0
    B = 3 * (m * xc).sum(axis=0) * xc / r ** 5 - m / r ** 3
    V = np.cross(E, B, axis=0) / (B ** 2).sum(axis=0)
    return V, xc / r


def test_ionospheric_ghosts(oracle_built):
    o, inE = _oracle()
    Gas, mf, xcc = o.array("Gas"), o.array("magFlux"), o.array("xyzcc")
    Nk, Nj = N[2] + 8, N[1] + 8
    kp = np.arange(Nk)
    kp = np.where(kp < G, kp + N[2], np.where(kp >= G + N[2], kp - N[2], kp))
    gamma = 5.0 / 3.0
    aj = slice(G, G + N[1])  # active j rows: the J boundary refills the others afterwards
    for n in range(1, 5):
        ig, ip = G - n, G + n - 1
        g = Gas[:, :, aj, ig]
        p = Gas[:, kp][:, :, aj, ip]
        rho_p = p[0]
        P_p = (gamma - 1) * (p[4] - 0.5 * (p[1] ** 2 + p[2] ** 2 + p[3] ** 2) / rho_p)
        assert np.allclose(g[0], np.maximum(rho_p, 1e-12), rtol=1e-13, atol=0)
        V, rh = _exb(xcc[:, kp][:, :, aj, ig], inE[:, kp][:, :, aj, 4 - n], dipole.M0)
        Vr = (V * rh).sum(axis=0)
        Vw = V - Vr * rh + np.minimum(Vr, 0.0) * rh
        Vg = g[1:4] / g[0]
        scale = np.abs(Vw).max()
        assert np.abs(Vg - Vw).max() <= 1e-11 * scale, np.abs(Vg - Vw).max() / scale
        assert ((Vg * rh).sum(axis=0) <= 1e-12 * scale).all()  # no outward radial velocity
        Pg = (gamma - 1) * (g[4] - 0.5 * (g[1] ** 2 + g[2] ** 2 + g[3] ** 2) / g[0])
        assert np.allclose(Pg, np.maximum(P_p, 1e-12), rtol=1e-10, atol=1e-14)
        assert (mf[0, :-1, :-1, ig] == 0).all() and (mf[1, :-1, :, ig] == 0).all() and (mf[2, :, :-1, ig] == 0).all()


def test_push_reaches_exb(oracle_built):
    o, inE = _oracle(dtCpl=1e-12)  # push factor min(dt / dtCpl, 1) = 1
    assert o.step(1) == 0
    Gas, xcc = o.array("Gas"), o.array("xyzcc")
    a = (slice(G, G + N[2]), slice(G, G + N[1]), G)
    g = Gas[(slice(None),) + a]
    V, rh = _exb(xcc[(slice(None),) + a], inE[:, G:G + N[2], G:G + N[1], 4], dipole.M0)
    Vp = V - (V * rh).sum(axis=0) * rh
    Vg = g[1:4] / g[0]
    assert np.abs(Vg - Vp).max() <= 1e-10 * np.abs(Vp).max()


def test_nudge_reaches_wind(oracle_built):
    o, _ = _oracle(dtSW0=1e-12)  # dtSW = max(dtSW0 / w, dt) = dt: the nudge factor is 1
    assert o.step(1) == 0
    w = dipole.wind_code_units()
    Gas, xcc = o.array("Gas"), o.array("xyzcc")
    ie = G + N[0] - 1
    g = Gas[:, G:G + N[2], G:G + N[1], ie]
    x = xcc[:, G:G + N[2], G:G + N[1], ie]
    V = np.asarray(w[2:5])
    # wgtWind (apps/wind.F90:180-203): full weight where the cell faces the wind
    cosang = -(V[:, None, None] * x).sum(axis=0) / (np.linalg.norm(V) * np.sqrt((x ** 2).sum(axis=0)))
    hit = cosang > 1e-3  # angle below 90 degrees: weight 1
    assert hit.any()
    assert np.allclose(g[0][hit], w[0], rtol=1e-12)
    for a in range(3):
        assert np.allclose((g[1 + a] / g[0])[hit], w[2 + a], rtol=1e-12, atol=1e-12)


def test_ionosphere_steps(oracle_built):
    o, _ = _oracle()
    assert o.step(5) == 0
    assert np.isfinite(o.array("Gas")).all()
    flux = np.abs(o.array("magFlux")).sum()
    assert o.divb() <= 1e-12 * flux
