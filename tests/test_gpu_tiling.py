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
