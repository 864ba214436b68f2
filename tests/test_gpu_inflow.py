"""Uniform inflow on the inner I side, zeroGrad_obcI (bcs.F90:820-850) on the
outer one, periodic J and K, through the C ABI (blast wave on the warped grid).

* strict build: initial fill and N steps identical, bit for bit, to the
  oracle built with the same erfc/exp;
* product FP64 build: <= 1e-12 relative to the oracle after 10 steps;
* the gradient of a loss w.r.t. the inflow state (mage_b200.diffstep with
  the hand-written CUDA stages) against central differences of the CUDA
  product step: <= 1e-5 relative per component.
"""
import numpy as np
import pytest
import torch

from mage_b200 import grids
from mage_b200.gamera import BC_INFLOW, BC_PERIODIC, BC_ZEROGRAD, GAM_ESTATE, GamError, GameraGPU, GamParams
from oracle.oracle import Oracle, OracleParams
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")
BCS = (BC_INFLOW, BC_ZEROGRAD, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC)
INFLOW = (1.0, 0.1, 0.5, 0.0, 0.0, 0.5 ** 0.5, 0.5 ** 0.5, 0.3)


def _pair(N, variant="gm", **kw):
    xyz = grids.warped_periodic_corners(*N)
    o = Oracle(OracleParams(*N, bc=BCS, inflow=INFLOW), xyz, variant)
    o.ic_blast_wave()
    assert o.init_finish() == 0
    g = GameraGPU(GamParams(*N, bc=BCS, **kw))
    g.set_geometry(xyz)
    g.set_inflow(INFLOW)
    g.init_blast_wave()
    return o, g


def test_inflow_strict_is_bit_exact(oracle_built):
    o, g = _pair((16, 12, 12), strict=True)
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), ("init", k, rel_err(s[k], o.array(k)))
    for nst in (1, 9):
        assert o.step(nst) == 0
        dt, t = g.step_gamera(nst)
        s = g.download_state()
        for k in STATE:
            assert np.array_equal(s[k], o.array(k)), (nst, k, rel_err(s[k], o.array(k)))
        assert dt == o.scalars()["dt"]


def test_inflow_product_build(oracle_built):
    o, g = _pair((32, 16, 16), variant="strict")
    assert o.step(10) == 0
    g.step_gamera(10)
    s = g.download_state()
    for k in ("Gas", "magFlux", "Bxyz"):
        assert rel_err(s[k], o.array(k)) <= 1e-12, (k, rel_err(s[k], o.array(k)))


def test_inflow_needs_its_state():
    N = (16, 8, 8)
    g = GameraGPU(GamParams(*N, bc=BCS))
    g.set_geometry(grids.warped_periodic_corners(*N))
    with pytest.raises(GamError) as e:
        g.init_blast_wave()
    assert e.value.code == GAM_ESTATE


def test_inflow_gradient_against_cuda_forward():
    from mage_b200.diffstep import DiffParams, Grid, loss_and_grad, win
    N, nst = (16, 8, 8), 6
    g0 = GameraGPU(GamParams(*N, bc=BCS))
    g0.set_geometry(grids.warped_periodic_corners(*N))
    g0.set_inflow(INFLOW)
    g0.init_blast_wave()
    st = g0.download_state(old=False)
    dt = 0.5 * st["dt"]
    gpu = GameraGPU(GamParams(*N, bc=BCS, fixedTimestep=dt))
    gpu.set_geometry(grids.warped_periodic_corners(*N))
    g = Grid(DiffParams(*N, bc=BCS), g0.get_geometry_arrays(), device="cuda", inflow=INFLOW)
    act = (4, 4 + N[0] - 1, 4, 4 + N[1] - 1, 4, 4 + N[2] - 1)
    mask = (win(g.xyzcc, act)[0] < 0.3).double()

    def lossf(gr, s):
        return ((win(s["B"], act) ** 2).sum(dim=0) * mask).sum()

    Gas0, mf0 = g.cell_box(st["Gas"]), g.face_box(st["magFlux"])
    L, gG, gF, (gp,) = loss_and_grad(g, Gas0, mf0, dt, nst, lossf=lossf, params=[g.inflow])
    Gas = np.ascontiguousarray(st["Gas"])
    mf = np.ascontiguousarray(st["magFlux"])
    with torch.no_grad():  # the start Bxyz of loss_and_grad: bFlux2Fld of the start fluxes
        B = np.ascontiguousarray(g.bxyz(mf0)[:, :g.Nk, :g.Nj, :g.Ni].cpu().numpy())

    def cuda_loss(w):
        gpu.set_inflow(w)
        gpu.upload_state(Gas, mf, B, Gas, mf, 0.0, -dt, dt, 0)
        gpu.step_gamera(nst)
        Bt = g.cell_box(gpu.download_state(old=False)["Bxyz"])
        return float(lossf(g, {"B": Bt}))

    assert abs(cuda_loss(np.asarray(INFLOW)) - L) <= 1e-12 * abs(L)
    base = np.asarray(INFLOW, dtype=np.float64)
    for q in (0, 1, 2, 7):  # rho, P, Vx, Bz
        e = np.zeros(8)
        e[q] = 1e-7 * max(abs(base[q]), 1.0)
        fd = (cuda_loss(base + e) - cuda_loss(base - e)) / (2 * e[q])
        assert abs(fd - float(gp[q])) <= 1e-5 * abs(float(gp[q])), (q, fd, float(gp[q]))
