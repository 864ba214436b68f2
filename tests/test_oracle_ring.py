"""The oracle's ring averaging about the LFM axis (ring/doRing with gid
"lfm": ringav.F90, ringrecon.F90, ringutils.F90, the pole boundaries lfmIn /
lfmOut of bcs.F90:1019-1106), checked on the CPU on a grid spherical about
the x axis (mage_b200.grids.lfm_corners):

* the pole boundaries: each ghost cell across the pole holds its conjugate's
  gas and Bxyz (mirrored j, k + Np/2), ghost I faces its flux, ghost J and K
  faces the negated flux;
* the ring average conserves the mass of every chunk, so a blast centred on
  the axis that has not reached the I boundaries keeps the total mass to
  round-off, and div B stays at round-off (the smoothing acts through an
  EMF);
* a state symmetric about the axis (a blast centred on it, no field) stays
  symmetric through a step and its ring average: the density is uniform
  along every ring to round-off. (The energy after one step, and everything
  after more steps, drift apart at 1e-5..1e-4 with or without rings: the
  limiters act on Cartesian velocity components, which are not invariant
  under rotation about the axis.)
"""
import numpy as np
import pytest

from mage_b200 import grids
from oracle.oracle import BC_LFM, BC_PERIODIC, BC_SPHIN, BC_ZEROGRAD, Oracle, OracleParams

N = (16, 16, 16)
BCS = (BC_SPHIN, BC_ZEROGRAD, BC_LFM, BC_LFM, BC_PERIODIC, BC_PERIODIC)


def _oracle(y0=0.0, nch=(8,), B0=0.3):
    o = Oracle(OracleParams(*N, bc=BCS, ringNch=nch), grids.lfm_corners(*N, th0=0.01), "strict")
    o.ic_blast_wave(x0=6.0, y0=y0, z0=0.0, rC=3.0, B0=B0)
    assert o.init_finish() == 0
    return o


def test_pole_ghosts_are_conjugates(oracle_built):
    o = _oracle(y0=1.0)
    assert o.step(2) == 0
    Gas, mf, B = o.array("Gas"), o.array("magFlux"), o.array("Bxyz")
    G, Njp, Np = 4, N[1], N[2]
    for n in range(1, 5):
        for jg, jc in ((G - n, G + n - 1), (G + Njp - 1 + n, G + Njp - n)):
            for k in range(Np + 8):
                kc = k + Np // 2
                if kc > G + Np - 1:
                    kc -= Np
                assert np.array_equal(Gas[:, k, jg, :], Gas[:, kc, jc, :]), (n, jg, k)
                assert np.array_equal(B[:, k, jg, :], B[:, kc, jc, :]), (n, jg, k)
                assert np.array_equal(mf[0, k, jg, :], mf[0, kc, jc, :])
                assert np.array_equal(mf[2, k, jg, :], -mf[2, kc, jc, :])
        # J faces: the pole face itself is not mirrored
        for k in range(Np + 8):
            kc = k + Np // 2
            if kc > G + Np - 1:
                kc -= Np
            assert np.array_equal(mf[1, k, G - n, :], -mf[1, kc, G + n, :])
            assert np.array_equal(mf[1, k, G + Njp + n, :], -mf[1, kc, G + Njp - n, :])


def test_mass_and_divb_kept(oracle_built):
    """The first step, before any flow reaches the I boundaries, keeps the
    total mass to round-off with the ring average acting; div B stays at
    round-off."""
    o = _oracle(y0=0.7)
    vol = o.array("volume")[0, 4:-4, 4:-4, 4:-4]
    m0 = float(np.sum(o.array("Gas")[0, 4:-4, 4:-4, 4:-4] * vol))
    assert o.step(1) == 0
    m = float(np.sum(o.array("Gas")[0, 4:-4, 4:-4, 4:-4] * vol))
    assert abs(m - m0) <= 1e-13 * m0, (m, m0)
    for _ in range(3):
        assert o.step(1) == 0
        assert o.divb() <= 1e-11


def test_axisymmetric_blast_stays_axisymmetric(oracle_built):
    o = _oracle(y0=0.0, B0=0.0)  # no field: the blast's uniform field is not along x
    assert o.step(1) == 0
    g = o.array("Gas")[:, 4:-4, 4:-4, 4:-4]  # (v, k, j, i)
    spread = np.max(np.abs(g - g.mean(axis=1, keepdims=True)), axis=(1, 2, 3))
    scale = np.max(np.abs(g), axis=(1, 2, 3))
    # the density; the momentum rotates with k, and the energy picks up the
    # limiters' response to Cartesian components
    assert spread[0] <= 1e-14 * scale[0], spread / scale


@pytest.mark.parametrize("nch", [(8,), (2, 4, 8)], ids=["1ring", "3rings"])
def test_ring_average_conserves_ring_sums_as_reference_test(oracle_built, nch):
    """The reference's own check of RingAverage (tests/voltron/testring.pf,
    ringAvgConservationTest), restated on this grid: the ring rows next to
    both poles get density 1 (k < ke/2) or 2, momenta sin(n k pi) times the
    density (n = 1, 2, 3) and fluxes sin(n k pi) (n = 4, 5, 6); one RingAverage
    alone keeps the density and momentum sum of every ring to 1e-15 and the
    total div B to 2e-13, the reference's tolerances."""
    o = _oracle(y0=1.0, nch=nch)
    assert o.step(1) == 0
    G, Njp, Nkp = 4, N[1], N[2]
    Gas, mf = o.array("Gas"), o.array("magFlux")
    NumR = len(nch)  # one ring per chunk count
    ks, ke = 1, Nkp
    rows = [G + r - 1 for r in range(1, NumR + 1)] + [G + Njp - r for r in range(1, NumR + 1)]
    for kf in range(ks, ke + 1):
        kk = kf - 1 + G
        den = 1.0 if kf < ke // 2 else 2.0
        for jj in rows:
            Gas[0, kk, jj, G:G + N[0]] = den
            for n in range(3):
                Gas[1 + n, kk, jj, G:G + N[0]] = np.sin((n + 1) * kf * np.pi) * den
            for d in range(3):
                mf[d, kk, jj, G:G + N[0]] = np.sin((4 + d) * kf * np.pi)
    before = {jj: Gas[0:4, G:G + Nkp, jj, G:G + N[0]].sum(axis=1) for jj in rows}
    den0 = Gas[0, G:G + Nkp, rows[0], G:G + N[0]].copy()
    div0 = o.divb()
    assert o.ring_average() == 0
    assert np.abs(Gas[0, G:G + Nkp, rows[0], G:G + N[0]] - den0).max() > 0.1  # the average acted
    for jj in rows:
        after = Gas[0:4, G:G + Nkp, jj, G:G + N[0]].sum(axis=1)
        assert np.abs(after - before[jj]).max() <= 1e-15, (jj, np.abs(after - before[jj]).max())
    assert abs(o.divb() - div0) <= 2e-13, (o.divb(), div0)


def test_metric_periodic_in_k_as_reference_test(oracle_built):
    """The reference's metric check on its LFM grid (tests/gamera/testfields.pf,
    testFaceMetricFields / testEdgeMetricFields), restated: with corners
    periodic in k (the k = ke+1.. layers copies of ks..), the K-face triads and
    areas at ks equal those at ke+1, and the I- and J-edge triads, edge maps
    and lengths at ks equal those at ke+1, exactly (the reference asserts a
    difference <= 0)."""
    G, Nip, Njp, Nkp = 4, N[0], N[1], N[2]
    xyz = grids.lfm_corners(*N, th0=0.01)
    # corner layer kk = G + Nkp + m repeats kk = G + m (and the lower ghosts the upper actives)
    for m in range(0, G + 1):
        xyz[:, G + Nkp + m] = xyz[:, G + m]
    for m in range(1, G + 1):
        xyz[:, G - m] = xyz[:, G + Nkp - m]
    o = Oracle(OracleParams(*N, bc=BCS, ringNch=(8,)), xyz, "strict")
    Tf, face, Te, Teb, edge = (o.array(n) for n in ("Tf", "face", "Te", "Teb", "edge"))
    a, b = G, G + Nkp  # ks and ke+1
    iA, jA = slice(G, G + Nip), slice(G, G + Njp)
    # K faces (d = 2) of the active cells
    assert np.array_equal(Tf[18:27, a, jA, iA], Tf[18:27, b, jA, iA])
    assert np.array_equal(face[2, a, jA, iA], face[2, b, jA, iA])
    # I edges (d = 0): i in is..ie, j in js..je+1; J edges (d = 1): i in is..ie+1, j in js..je
    iE, jE = slice(G, G + Nip), slice(G, G + Njp + 1)
    assert np.array_equal(Te[0:9, a, jE, iE], Te[0:9, b, jE, iE])
    assert np.array_equal(Teb[0:4, a, jE, iE], Teb[0:4, b, jE, iE])
    assert np.array_equal(edge[0, a, jE, iE], edge[0, b, jE, iE])
    iE, jE = slice(G, G + Nip + 1), slice(G, G + Njp)
    assert np.array_equal(Te[9:18, a, jE, iE], Te[9:18, b, jE, iE])
    assert np.array_equal(Teb[4:8, a, jE, iE], Teb[4:8, b, jE, iE])
    assert np.array_equal(edge[1, a, jE, iE], edge[1, b, jE, iE])
