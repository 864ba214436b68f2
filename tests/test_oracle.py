"""CPU tests of the oracle (the CPU restatement of the reference step):
pinned against the reference's own known-answer tests and invariants."""
import json
import os

import numpy as np
import pytest

from mage_b200 import grids
from oracle import oracle as orc
from tests.helpers import make_oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _frac(s):
    if isinstance(s, str) and "/" in s:
        a, b = s.split("/")
        return float(a) / float(b)
    return float(s)


@pytest.mark.parametrize("variant", ["strict", "gm"])
def test_gamutils_kat(oracle_built, variant):
    """tests/gamera/testgamutils.pf:24-112 (CellP2C / CellC2P known answers)."""
    k = json.load(open(os.path.join(GOLD, "gamutils_kat.json")))
    gamma = _frac(k["gamma"])
    prim = np.array([_frac(x) for x in k["prim"]])
    con = np.array(k["con"])
    c = orc.p2c(prim, gamma, variant)
    assert np.all(np.abs(c - con) <= np.array(k["p2c_tol"]))
    p = orc.c2p(con, gamma, variant)
    assert np.all(np.abs(p - prim) <= np.array(k["c2p_tol"]))
    c2 = orc.p2c(orc.c2p(con, gamma, variant), gamma, variant)
    assert np.all(np.abs(c2 - con) <= np.array(k["c2c_tol"]))
    p2 = orc.c2p(orc.p2c(prim, gamma, variant), gamma, variant)
    assert np.all(np.abs(p2 - prim) <= np.array(k["p2p_tol"]))


def test_metric_box(oracle_built):
    """tests/gamera/testmetric.pf: the box (1,1,1)-(2,3,4) as cell (1,1,1) of a
    uniform grid; the quadrature metric reproduces its centre, face centres and
    areas (Corners2Grid, init.F90:793-1072)."""
    m = json.load(open(os.path.join(GOLD, "metric_kat.json")))
    xyz = grids.uniform_corners(16, 4, 4, bounds=(1.0, 17.0, 1.0, 9.0, 1.0, 13.0))
    o = orc.Oracle(orc.OracleParams(16, 4, 4), xyz)
    c = (slice(None), 4, 4, 4)  # Fortran (1,1,1) -> box index 4 (isg = -3)
    assert np.allclose(o.array("xyzcc")[c], m["cell_center"], rtol=0, atol=1e-13)
    xfc = o.array("xfc")[c].reshape(3, 3)  # [d][x]
    for d, name in enumerate("IJK"):
        assert np.allclose(xfc[d], m["face_center"][name], rtol=0, atol=1e-13)
    face = o.array("face")[c]
    assert np.allclose(face, [6.0, 3.0, 2.0], rtol=1e-14)
    assert abs(o.array("volume")[0, 4, 4, 4] - 6.0) < 1e-13
    # corner array of the box matches the reference corner ordering
    for d, name in enumerate("IJK"):
        f = m["face_coords"][name]
        assert np.allclose(xyz[:, 4, 4, 4], f[0])
    # face triads are orthonormal, normal along the face direction
    Tf = o.array("Tf")[c].reshape(3, 3, 3)  # [d][vec][x]
    for d in range(3):
        assert np.allclose(Tf[d] @ Tf[d].T, np.eye(3), atol=1e-14)
        assert abs(Tf[d][0][d] - 1.0) < 1e-14


def _ulps(a, ref):
    import mpmath as mp  # noqa: F401  (only needed for the string refs)
    ref = float(ref)
    if ref == 0.0:
        return 0.0 if a == 0.0 else np.inf
    return abs(a - ref) / np.spacing(abs(ref))


def test_erfc_exp_golden(oracle_built):
    """Self-written FP64 erfc/exp (mage_b200/csrc/gam_math.cuh, via the 'gm'
    oracle build) against 40-digit reference values: <= 8 ulp for erfc,
    <= 2 ulp for exp, in the normal range."""
    g = json.load(open(os.path.join(GOLD, "erfc_exp.json")))
    L = orc.lib("gm")
    for xh, ref in g["erfc"]:
        x = float.fromhex(xh)
        r = float(ref)
        if r < 1e-300:
            continue
        assert _ulps(L.orc_erfc(x), ref) <= 8.0, (x, L.orc_erfc(x), ref)
    for xh, ref in g["exp"]:
        x = float.fromhex(xh)
        r = float(ref)
        if r < 1e-300 or r > 1e300:
            continue
        assert _ulps(L.orc_exp(x), ref) <= 2.0, (x, L.orc_exp(x), ref)


def ot_symmetry(Gas, N):
    """Symmetry violation of the Orszag-Tang state, tests/cases/testCases.pf:198-216."""
    G = Gas[:, 4, 4:4 + N, 4:4 + N]  # k = ks slice, active (j, i)
    F = G[:, ::-1, ::-1].copy()
    F[1:3] *= -1.0
    return float(np.sqrt(((G - F) ** 2).sum(axis=0)).sum() / (N * N))


@pytest.mark.parametrize("Nk", [1, 4])
def test_ot_symmetry(oracle_built, Nk):
    """OT point symmetry (testCases.pf:183-225 asserts <= 1e-11)."""
    N = 32
    o, _ = make_oracle("ot", (N, N, Nk))
    assert o.step(40) == 0
    assert ot_symmetry(o.array("Gas"), N) <= 1e-11


def test_conservation_and_divb(oracle_built):
    """Periodic curvilinear blast wave: mass and Cartesian momentum are
    conserved to round-off (the fluxes telescope), div B stays at round-off
    (DivB, gridutils.F90:717-770). Plasma energy is not conserved by itself:
    CellMaxwell (mhdgroup.F90:299-329) exchanges it with the field."""
    o, _ = make_oracle("bw", (16, 16, 16))
    vol = o.array("volume")[0, 4:-4, 4:-4, 4:-4]

    def tot():
        G = o.array("Gas")[:, 4:-4, 4:-4, 4:-4]
        return np.array([(G[v] * vol).sum() for v in range(5)])

    t0 = tot()
    phi = np.abs(o.array("magFlux")).sum()
    assert o.step(10) == 0
    t1 = tot()
    assert abs(t1[0] - t0[0]) / t0[0] < 1e-13
    mscale = np.abs(o.array("Gas")[1:4, 4:-4, 4:-4, 4:-4] * vol).sum()
    assert np.abs(t1[1:4] - t0[1:4]).max() < 1e-13 * mscale
    assert o.divb() < 1e-12 * phi


def test_variants_agree(oracle_built):
    """libm erfc/exp vs the self-written ones vs -ffast-math: the same step to
    well below 1e-12 after 20 steps."""
    ref, _ = make_oracle("ot", (32, 32, 4), "strict")
    ref.step(20)
    for v in ("gm", "fast"):
        o, _ = make_oracle("ot", (32, 32, 4), v)
        o.step(20)
        a, b = o.array("Gas"), ref.array("Gas")
        assert np.abs(a - b).max() / np.abs(b).max() < 1e-12


def test_dt_limit_is_reported(oracle_built):
    """CalcDT flags a timestep below limDT0*dt0 as bad (step.F90:117-121)
    instead of continuing."""
    o, _ = make_oracle("ot", (32, 32, 4))
    assert o.step(2) == 0
    o.set_scalars(dt0=1.0e5 * o.scalars()["dt"])
    assert o.step(1) == 1  # ST_DT_BAD


def test_boris_limits(oracle_built):
    """Boris correction in the oracle: with Ca -> HUGE it reduces to the step
    without it (the Boris speed, Vac2 and CellBoris's alpha vanish; only
    rounding differs), and a Ca below the flow speeds changes the solution
    (Boris-limited speeds, hogs, the nuclear option) while keeping mass and
    divB exact."""
    N = (32, 32, 4)
    xyz = grids.uniform_corners(*N)

    def run(**kw):
        o = orc.Oracle(orc.OracleParams(*N, **kw), xyz, "strict")
        o.ic_orszag_tang()
        assert o.init_finish() == 0
        assert o.step(10) == 0
        return o

    a, b, c = run(), run(doBoris=True, Ca=1.0e12), run(doBoris=True, Ca=0.5)
    ga, gb, gc = a.array("Gas"), b.array("Gas"), c.array("Gas")
    act = (slice(None), slice(4, 8), slice(4, 36), slice(4, 36))
    assert np.abs(gb - ga).max() <= 1e-12 * np.abs(ga).max()
    d = float(np.abs(gc[act] - ga[act]).max() / np.abs(ga[act]).max())
    assert d > 1e-3, d
    m0 = a.array("Gas")[0][act[1:]].sum()
    assert abs(gc[0][act[1:]].sum() - m0) <= 1e-12 * m0
    assert c.divb() <= 1e-12 * np.abs(c.array("magFlux")).sum()


def test_ab3_predictor(oracle_built):
    """AB3 (mhdgroup.F90:444-517, 721-731) in the oracle: its first step from
    the start (State = oState = ooState) equals AB2's bit for bit, later steps
    differ at the scheme's truncation level, and ooState trails oState by one
    step in time."""
    N = (16, 16, 16)
    xyz = grids.warped_periodic_corners(*N)

    def run(nst, **kw):
        o = orc.Oracle(orc.OracleParams(*N, **kw), xyz, "strict")
        o.ic_blast_wave()
        assert o.init_finish() == 0
        assert o.step(nst) == 0
        return o

    a1, b1 = run(1), run(1, doAB3=True)
    assert np.array_equal(a1.array("Gas"), b1.array("Gas"))
    a, b = run(10), run(10, doAB3=True)
    d = float(np.linalg.norm(b.array("Gas") - a.array("Gas")) / np.linalg.norm(a.array("Gas")))
    assert 0 < d < 1e-2, d
    sc = b.scalars()
    assert sc["ootime"] < sc["otime"] < sc["time"]


def _dipole_oracle(N=(16, 8, 8), series=None):
    from mage_b200 import dipole
    w = dipole.wind_code_units()
    o = orc.Oracle(orc.OracleParams(*N, doBackground=True, M0=dipole.M0, wind=w, bc=(3, 4, 2, 2, 0, 0)),
                   grids.spherical_corners(*N), "strict")
    o.ic_dipole_wind(0.01, 31337)
    if series is not None:
        o.set_wind_series(**series)
    assert o.init_finish() == 0
    return o, w


def test_wind_series_restates_the_constant_wind(oracle_built):
    """A time series (apps/wind.F90:116-203, 766-868) whose rows all hold the
    constant wind, with Bx0 = Bx and ByC = BzC = 0 so that readWind's tilted
    front (Bx = Bx0 + ByC By + BzC Bz) keeps Bx, steps exactly like the
    constant wind; a series that changes after 2 time units differs."""
    from mage_b200 import dipole
    w = dipole.wind_code_units()
    # rows cover every lag time of the grid (|DelT| <= 30 / 4 here), so no
    # point sees the null field of times before the series
    n = 21
    t = np.linspace(-100.0, 100.0, n)
    const = dict(t=t, rho=np.full(n, w[0]), P=np.full(n, w[1]), V=np.tile(w[2:5], (n, 1)),
                 B=np.tile(w[5:8], (n, 1)), Bx0=w[5])
    a, _ = _dipole_oracle()
    b, _ = _dipole_oracle(series=const)
    assert a.step(5) == 0 and b.step(5) == 0
    for k in ("Gas", "magFlux", "Bxyz"):
        assert np.array_equal(a.array(k), b.array(k)), k
    # a denser wind from t = 0 on: the ghost shell changes
    var = dict(const)
    rho = const["rho"].copy()
    rho[t >= 0.0] *= 2.0
    var["rho"] = rho
    c, _ = _dipole_oracle(series=var)
    assert c.step(1) == 0
    a1, _ = _dipole_oracle()
    assert a1.step(1) == 0
    assert not np.array_equal(a1.array("Gas"), c.array("Gas"))


@pytest.mark.parametrize("up7", [True, False], ids=["7UP", "8CENT"])
def test_reference_adv1d_case(oracle_built, up7):
    """tests/cases/testCases.pf:114-180 (testAdv1D, testAdv1D_8CENT) with its
    decks adv1d.xml / adv1d_8cent.xml: hydro (gamma 1.4 from initADV1D,
    prob.F90:671-736), pdmb 4 (so CFL = 0.5/4.5), 128 cells on [-1, 1], one
    advection period (tFin 2); L2 = norm2(start - end density) / Nip <= 7e-3."""
    N = (128, 1, 1)
    xyz = grids.uniform_corners(*N, bounds=(-1.0, 1.0, -0.5, 0.5, -0.5, 0.5))
    o = orc.Oracle(orc.OracleParams(*N, doMHD=False, gamma=1.4, pdmb=4.0, CFL=min(0.5 / 4.5, 0.3), up7=up7, tFin=2.0),
                   xyz, "strict")
    o.ic_case("adv1d")
    assert o.init_finish() == 0
    sD = o.array("Gas")[0, 4, 4, 4:132].copy()
    while o.scalars()["t"] < 2.0:
        assert o.step(1) == 0
    L2 = float(np.linalg.norm(sD - o.array("Gas")[0, 4, 4, 4:132]) / 128)
    assert L2 <= 7.0e-3, L2
