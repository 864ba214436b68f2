"""k-slab tiling on one GPU: the slabs of mage_b200.tiling.Slabs, kept in one
process and swapping halos by device copies, against the periodic
single-domain step. Every value a step defines (active cells, ghosts, faces)
is identical bit for bit, with 1 slab (halo sent to itself) and with 2 and 4
slabs, for the product and the strict build."""
import numpy as np
import pytest

from mage_b200 import grids
from mage_b200.gamera import GameraGPU, GamParams
from mage_b200.tiling import Slabs

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
