"""Tiling on one GPU: the tiles of mage_b200.tiling.Slabs / Tiles, kept in one
process and swapping halos by device copies, against the single-domain step.
Every value a step defines (active cells, ghosts, faces) is identical bit for
bit: k-slabs (1 slab with its halo sent to itself, 2 and 4 slabs), tiles along
two and three directions of the periodic blast wave, and the magnetosphere
(ionospheric boundary, wind and their hooks) cut in i and j; for the product
and the strict build. The exchange alone is checked on affine data."""
import numpy as np
import pytest

from mage_b200 import grids
from mage_b200.gamera import (BC_HALO, BC_ION, BC_PERIODIC, BC_WIND, BC_ZEROGRAD, GameraGPU,
                              GamParams)
from mage_b200.tiling import Slabs, Tiles, tile_box, tile_cut

pytestmark = pytest.mark.gpu


def _compare(slabs, ref, nk):
    for r, g in zip(slabs.ranks, slabs.apps):
        s = g.download_state()
        k0 = r * nk
        for name in ("Gas", "Bxyz", "oGas"):
            assert np.array_equal(s[name], ref[name][:, k0:k0 + nk + 8]), (r, name)
        for name in ("magFlux", "omagFlux"):
            a, b = s[name], ref[name][:, k0:k0 + nk + 9]
            assert np.array_equal(a[:2, :nk + 8], b[:2, :nk + 8]), (r, name, "I/J faces")
            assert np.array_equal(a[2], b[2]), (r, name, "K faces")
        assert s["dt"] == ref["dt"] and s["time"] == ref["time"] and s["ts"] == ref["ts"]


@pytest.mark.parametrize("nslab,strict", [(1, False), (2, False), (4, False), (2, True)])
def test_slabs_equal_single_domain(nslab, strict):
    N = (16, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    one = GameraGPU(GamParams(*N, strict=strict))
    one.set_geometry(xyz)
    one.init_blast_wave()
    sl = Slabs(N, xyz, nslab, strict=strict)
    _compare(sl, one.download_state(), N[2] // nslab)
    for n in (1, 6):
        dt1, t1 = one.step_gamera(n)
        dt2, t2 = sl.step(n)
        assert (dt1, t1) == (dt2, t2)
        _compare(sl, one.download_state(), N[2] // nslab)


@pytest.mark.parametrize("nslab", [2, 4])
def test_affine_halo_exchange(nslab):
    """The halo exchange alone, in the manner of the reference's MPI halo test
    (tests/gamera_mpi/testmpimhd.pf:44-160): every value of every slab holds an
    affine function of its component and its global (i, j, k) index, periodic
    in k; the k ghost layers start as a sentinel. After one exchange (with
    Bxyz copied, as in the first fill) each ghost holds exactly the value at
    its wrapped global index, and no active value changed."""
    N = (16, 8, 16)
    nk = N[2] // nslab
    sl = Slabs(N, grids.warped_periodic_corners(*N), nslab)
    lv, iv, jv, kv = 1.0e9, 1.0, 1.0e3, 1.0e6
    SENT = -7.0e20

    def affine(nc, face, r, q0):
        Ni, Nj = N[0] + 8, N[1] + 8
        Nk = nk + 8 + (1 if face else 0)
        kk = np.arange(Nk)
        kg = np.mod(r * nk + kk - 4, N[2]).astype(np.float64)
        ii = np.arange(Ni + (1 if face else 0), dtype=np.float64)
        jj = np.arange(Nj + (1 if face else 0), dtype=np.float64)
        a = (lv * (q0 + np.arange(nc))[:, None, None, None] + kv * kg[None, :, None, None] +
             jv * jj[None, None, :, None] + iv * ii[None, None, None, :])
        return a

    ref = {}
    for r, g in zip(sl.ranks, sl.apps):
        A = {"Gas": affine(5, False, r, 0), "magFlux": affine(3, True, r, 5), "Bxyz": affine(3, False, r, 8)}
        ref[r] = {k: v.copy() for k, v in A.items()}
        for k, v in A.items():  # the k ghosts start as a sentinel
            v[:, :4] = SENT
            v[:, nk + 4:] = SENT
        A["magFlux"][2, nk + 4] = ref[r]["magFlux"][2, nk + 4]  # the slab's own upper K face is active
        g.upload_state(A["Gas"], A["magFlux"], A["Bxyz"], A["Gas"], A["magFlux"], 0.0, -1.0, 1.0, 0)
    sl.exchange(copyB=True)
    for r, g in zip(sl.ranks, sl.apps):
        s = g.download_state()
        for k in ("Gas", "Bxyz"):
            assert np.array_equal(s[k], ref[r][k]), (r, k)
        mf, want = s["magFlux"], ref[r]["magFlux"]
        # I and J faces on the cell layers; K faces on 0..3 and nk+5..nk+8 (face
        # nk+4 is the slab's own upper active face)
        assert np.array_equal(mf[:2, :nk + 8], want[:2, :nk + 8]), r
        assert np.array_equal(mf[2, :4], want[2, :4]) and np.array_equal(mf[2, nk + 5:], want[2, nk + 5:]), r
        assert np.array_equal(mf[:, 4:nk + 5], want[:, 4:nk + 5]), r


# --- tiles along i, j and k ---------------------------------------------------------
def _box_equal(a, b, face: bool):
    """Every value of a box array that exists: cells whole; face component d
    over the face-box slots of faces normal to d."""
    if not face:
        return np.array_equal(a, b)
    ok = np.array_equal(a[0][:-1, :-1, :], b[0][:-1, :-1, :])
    ok = ok and np.array_equal(a[1][:-1, :, :-1], b[1][:-1, :, :-1])
    return ok and np.array_equal(a[2][:, :-1, :-1], b[2][:, :-1, :-1])


def _compare_tiles(tl, ref):
    for t, g in zip(tl.tiles, tl.apps):
        s = g.download_state()
        for name in ("Gas", "Bxyz", "oGas"):
            assert np.array_equal(s[name], tile_box(ref[name], tl.N, tl.dims, t.t)), (t.t, name)
        for name in ("magFlux", "omagFlux"):
            assert _box_equal(s[name], tile_box(ref[name], tl.N, tl.dims, t.t), True), (t.t, name)
        assert s["dt"] == ref["dt"] and s["time"] == ref["time"] and s["ts"] == ref["ts"]


@pytest.mark.parametrize("dims,strict", [((2, 2, 1), True), ((2, 1, 2), False), ((2, 2, 2), False),
                                         ((1, 2, 2), True)])
def test_tiles_equal_single_domain(dims, strict):
    """Periodic blast wave cut into tiles along two or three directions: the
    halo exchange I, then J, then K fills faces, edges and corners, and every
    value of every tile equals the single grid's, ghosts included."""
    N = (32, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    one = GameraGPU(GamParams(*N, strict=strict))
    one.set_geometry(xyz)
    one.init_blast_wave()
    tl = Tiles(N, xyz, dims, strict=strict)
    _compare_tiles(tl, one.download_state())
    for n in (1, 6):
        assert one.step_gamera(n) == tl.step(n)
        _compare_tiles(tl, one.download_state())


def test_affine_halo_exchange_three_directions():
    """The exchange alone on 2 x 2 x 2 tiles (periodic): every value holds an
    affine function of its component and wrapped global (i, j, k) index, the
    ghosts start as a sentinel; after one exchange (Bxyz copied) every ghost,
    edges and corners included, holds the value at its wrapped global index."""
    N, dims = (32, 16, 16), (2, 2, 2)
    tl = Tiles(N, grids.warped_periodic_corners(*N), dims)
    n = tl.n
    SENT = -7.0e20

    def affine(nc, face, t, q0):
        ax = []
        for d in range(3):
            x = np.arange(n[d] + 8 + (1 if face else 0))
            ax.append(np.mod(t[d] * n[d] + x - 4, N[d]).astype(np.float64))
        return (1.0e9 * (q0 + np.arange(nc))[:, None, None, None] + 1.0e6 * ax[2][None, :, None, None] +
                1.0e3 * ax[1][None, None, :, None] + ax[0][None, None, None, :])

    def ghost_mask(face, comp):
        m = np.zeros(tuple(n[d] + 8 + (1 if face else 0) for d in (2, 1, 0)), dtype=bool)
        for d, axis in ((0, 2), (1, 1), (2, 0)):
            top = 4 + n[d] + (1 if face and comp == d else 0)  # a tile's own upper face is active
            sl = [slice(None)] * 3
            sl[axis] = slice(0, 4)
            m[tuple(sl)] = True
            sl[axis] = slice(top, None)
            m[tuple(sl)] = True
        return m

    ref = {}
    for t, g in zip(tl.tiles, tl.apps):
        A = {"Gas": affine(5, False, t.t, 0), "magFlux": affine(3, True, t.t, 5), "Bxyz": affine(3, False, t.t, 8)}
        ref[t.t] = {k: v.copy() for k, v in A.items()}
        for k, v in A.items():
            for q in range(v.shape[0]):
                v[q][ghost_mask(k == "magFlux", q)] = SENT
        g.upload_state(A["Gas"], A["magFlux"], A["Bxyz"], A["Gas"], A["magFlux"], 0.0, -1.0, 1.0, 0)
    tl.exchange(copyB=True)
    for t, g in zip(tl.tiles, tl.apps):
        s = g.download_state()
        for k in ("Gas", "Bxyz"):
            assert np.array_equal(s[k], ref[t.t][k]), (t.t, k)
        assert _box_equal(s["magFlux"], ref[t.t]["magFlux"], True), t.t


MBCS = (BC_ION, BC_WIND, BC_ZEROGRAD, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC)


@pytest.mark.parametrize("push", [True, False], ids=["push", "nopush"])
def test_magnetosphere_tiles_equal_single_domain(push):
    """The dipole in the solar wind with the ionospheric inner boundary and its
    hooks, cut into 2 x 2 tiles in i and j (the decomposition the reference
    runs the magnetosphere with; k stays whole): the inner tiles hold the
    boundary, IonEFix and PushIon, the outer ones the wind, WindEFix and
    NudgeSW, all of them FixEFieldLFM and the active-cell DT range. From the
    single grid's state after 2 steps, every value of every tile equals the
    single grid's after 1 and 6 more steps (strict build)."""
    from mage_b200 import dipole
    N, dims = (32, 16, 8), (2, 2, 1)
    wind = dipole.wind_code_units()
    dtcpl = 5.0 / 63.8
    xyz = grids.spherical_corners(*N)
    rng = np.random.default_rng(7)
    E = 200.0 * rng.standard_normal((3, N[2] + 8, N[1] + 8, 5))
    Ee = 200.0 * rng.standard_normal((3, N[2] + 9, N[1] + 9, 6))
    one = GameraGPU(GamParams(*N, doBackground=1, bc=MBCS, strict=True))
    one.set_geometry(xyz)
    one.set_background_dipole(dipole.M0)
    one.set_ionosphere(E, Ee, dipole.M0, dtcpl, push, 2)
    one.init_dipole_wind(wind, 31337, 0.01)
    one.step_gamera(2)
    s0 = one.download_state()

    def setup(g, t):
        g.set_background_dipole(dipole.M0)
        if t.bc[1] == BC_WIND:
            g.set_wind(wind)
        if t.bc[0] == BC_ION:
            g.set_ionosphere(tile_cut(E, 2, N[1], dims[1], t.t[1]), tile_cut(Ee, 2, N[1], dims[1], t.t[1]),
                             dipole.M0, dtcpl, push, 2)
        else:
            g.set_ionosphere(None, None, dipole.M0, dtcpl, push, 2)
        st = {k: tile_box(s0[k], N, dims, t.t) for k in ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")}
        g.upload_state(st["Gas"], st["magFlux"], st["Bxyz"], st["oGas"], st["omagFlux"], s0["time"], s0["otime"],
                       s0["dt"], s0["ts"])

    tl = Tiles(N, xyz, dims, strict=True, bc=MBCS, problem=setup, params={"doBackground": 1})
    assert [t.bc for t in tl.tiles][:2] == [(BC_ION, BC_HALO, BC_ZEROGRAD, BC_HALO, BC_PERIODIC, BC_PERIODIC),
                                          (BC_HALO, BC_WIND, BC_ZEROGRAD, BC_HALO, BC_PERIODIC, BC_PERIODIC)]
    for n in (1, 6):
        assert one.step_gamera(n) == tl.step(n)
        _compare_tiles(tl, one.download_state())
