"""The non-periodic I boundaries of the differentiation form as kernels
(gam_iside_fill / gam_iside_adjoint: the uniform inflow or SphIn on the
inner side, zeroGrad_obcI or the constant solar wind on the outer side)
and the whole step with them (gam_step_fwd_save_iside / gam_step_adj_iside):

* the fill equals its PyTorch restatement (mage_b200.diffstep._iside_bcs)
  to <= 1e-14 relative (FP64; the kernel contracts products into fmas) and
  <= 1e-6 (FP32);
* the adjoint (of the state, of the field the outer fills read and of the
  inflow state) equals torch.autograd.grad through the restatement to
  <= 1e-12 relative L2 in FP64;
* the whole step equals step() bit for bit and its adjoint equals autograd
  through step() to <= 1e-12 (FP64) / 1e-5 (FP32), the same bits on every
  call, with the inflow state's gradient; the checkpointed C sweep gives the
  loss and the gradients (state and inflow) of loss_and_grad.
"""
import numpy as np
import pytest
import torch

from mage_b200 import dipole, grids
from mage_b200.diffstep import (DiffParams, Grid, WholeStep, _ISideFn, _iside_bcs, loss_and_grad, loss_and_grad_c,
                                step, win)
from mage_b200.gamera import GameraGPU, GamParams
from mage_b200.workloads import DIPOLE_BCS

pytestmark = pytest.mark.gpu

INFLOW_BCS = (6, 2, 0, 0, 0, 0)
INFLOW = (1.0, 0.1, 0.5, 0.0, 0.0, 0.5 ** 0.5, 0.5 ** 0.5, 0.3)


def _setup(kind, dtype, seed):
    """Grid and a noisy start of the dipole in the wind (SphIn, wind,
    zero-gradient J) or of the blast wave with the inflow (inflow, obcI)."""
    if kind == "dipole":
        N = (16, 8, 8)
        w = dipole.wind_code_units()
        gpu = GameraGPU(GamParams(*N, doBackground=True, bc=DIPOLE_BCS))
        gpu.set_geometry(grids.spherical_corners(*N))
        gpu.set_background_dipole(dipole.M0)
        gpu.init_dipole_wind(w)
        st = gpu.download_state(old=False)
        g = Grid(DiffParams(*N, bc=DIPOLE_BCS), gpu.get_geometry_arrays(), background=gpu.get_background(),
                 wind=w, dtype=dtype, device="cuda")
    else:
        N = (16, 16, 16)
        gpu = GameraGPU(GamParams(*N, bc=INFLOW_BCS))
        gpu.set_geometry(grids.warped_periodic_corners(*N))
        gpu.set_inflow(INFLOW)
        gpu.init_blast_wave()
        st = gpu.download_state(old=False)
        g = Grid(DiffParams(*N, bc=INFLOW_BCS), gpu.get_geometry_arrays(), dtype=dtype, device="cuda",
                 inflow=INFLOW)
    rng = np.random.default_rng(seed)
    shp = (5,) + tuple(g.face.shape[1:])
    Gas0 = g.cell_box(st["Gas"]) * (1 + 1e-3 * torch.as_tensor(rng.standard_normal(shp), device="cuda").to(dtype))
    mf0 = g.face_box(st["magFlux"]) + 1e-3 * g.face * torch.as_tensor(rng.standard_normal(g.face.shape),
                                                                       device="cuda").to(dtype)
    dt = 0.25 * st["dt"]
    return g, Gas0, mf0, dt, rng


def _rel(a, b):
    num = sum(float((x - y).double().norm()) ** 2 for x, y in zip(a, b)) ** 0.5
    den = sum(float(y.double().norm()) ** 2 for y in b) ** 0.5
    return num / den


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-14), (torch.float32, 1e-6)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["dipole", "inflow"])
def test_fill_matches_restatement(kind, dtype, tol):
    g, Gas, mf, _, _ = _setup(kind, dtype, 3)
    B = g.bxyz(mf)
    with torch.no_grad():
        rG, rM = _iside_bcs(g, Gas, mf, B)
        cG, cM = _ISideFn.apply(Gas, mf, B, g.inflow, g)
    for c, r in ((cG, rG), (cM, rM)):
        err = float((c - r).abs().max() / r.abs().max())
        assert err <= tol, err
    # the fill leaves every position it does not own as it was
    own = torch.zeros_like(Gas[0], dtype=torch.bool)
    own[..., :4] = True
    own[..., 4 + g.P.Nip:] = True
    assert torch.equal(cG[:, ~own], Gas[:, ~own])


@pytest.mark.parametrize("kind", ["dipole", "inflow"])
def test_adjoint_matches_autograd(kind):
    g, Gas, mf, _, rng = _setup(kind, torch.float64, 4)
    B = g.bxyz(mf)
    leaves = [t.detach().clone().requires_grad_(True) for t in (Gas, mf, B)]
    ws = [g.inflow.detach().clone().requires_grad_(True)] if g.inflow is not None else []
    dG = torch.as_tensor(rng.standard_normal(Gas.shape), device="cuda")
    dM = torch.as_tensor(rng.standard_normal(mf.shape), device="cuda")
    keep = g.inflow
    with torch.enable_grad():
        if ws:
            g.inflow = ws[0]
        try:
            rG, rM = _iside_bcs(g, *leaves)
            ref = torch.autograd.grad([rG, rM], leaves + ws, [dG, dM])
            cl = [t.detach().clone().requires_grad_(True) for t in (Gas, mf, B)] + \
                 [w.detach().clone().requires_grad_(True) for w in ws]
            cG, cM = _ISideFn.apply(cl[0], cl[1], cl[2], cl[3] if ws else None, g)
            got = torch.autograd.grad([cG, cM], cl, [dG, dM])
        finally:
            g.inflow = keep
    assert _rel(got[:3], ref[:3]) <= 1e-12, _rel(got[:3], ref[:3])
    if ws:
        assert _rel(got[3:], ref[3:]) <= 1e-12, (got[3], ref[3])


def _pair(g, Gas0, mf0, dt):
    with torch.no_grad():
        old = {"Gas": Gas0, "mf": mf0, "B": g.bxyz(mf0)}
        cur = step(g, old, old, dt, dt)
    return cur, old


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["dipole", "inflow"])
def test_whole_step_forward(kind, dtype):
    g, Gas0, mf0, dt, _ = _setup(kind, dtype, 5)
    cur, old = _pair(g, Gas0, mf0, dt)
    with torch.no_grad():
        ref = step(g, cur, old, dt, dt)
    out = WholeStep(g).forward(cur, old, dt, dt)
    for k in ("Gas", "mf", "B"):
        assert torch.equal(out[k], ref[k]), (k, float((out[k] - ref[k]).abs().max()))


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["dipole", "inflow"])
def test_whole_step_adjoint(kind, dtype, tol):
    g, Gas0, mf0, dt, rng = _setup(kind, dtype, 7)
    cur, old = _pair(g, Gas0, mf0, dt)
    leaves = [t.detach().clone().requires_grad_(True) for t in (cur["Gas"], cur["mf"], old["Gas"], old["mf"])]
    ws = [g.inflow.detach().clone().requires_grad_(True)] if g.inflow is not None else []
    keep = g.inflow
    with torch.enable_grad():
        if ws:
            g.inflow = ws[0]
        try:
            c = {"Gas": leaves[0], "mf": leaves[1], "B": g.bxyz(leaves[1])}
            o = {"Gas": leaves[2], "mf": leaves[3], "B": g.bxyz(leaves[3])}
            out = step(g, c, o, dt, dt)
            dn = {k: torch.as_tensor(rng.standard_normal(out[k].shape), device="cuda").to(dtype) for k in out}
            ref = torch.autograd.grad([out[k] for k in ("Gas", "mf", "B")], leaves + ws,
                                      [dn[k] for k in ("Gas", "mf", "B")])
        finally:
            g.inflow = keep
    wst = WholeStep(g)
    dw = torch.zeros(8, dtype=dtype, device="cuda") if ws else None
    got = wst.adjoint(cur, old, dt, dt, dn, dinflow=dw)
    assert _rel(got, ref[:4]) <= tol, _rel(got, ref[:4])
    if ws:
        assert _rel([dw], ref[4:]) <= tol, (dw, ref[4])
    wst.forward(cur, old, dt, dt)
    dw2 = torch.zeros_like(dw) if ws else None
    got2 = wst.adjoint(cur, old, dt, dt, dn, saved=True, dinflow=dw2)
    for a, b in zip(got2, got):
        assert torch.equal(a, b), float((a - b).abs().max())
    if ws:
        assert torch.equal(dw2, dw)


def test_sweep_with_inflow_gradient():
    g, Gas0, mf0, dt, _ = _setup("inflow", torch.float64, 11)
    act = (4, 4 + g.P.Nip - 1, 4, 4 + g.P.Njp - 1, 4, 4 + g.P.Nkp - 1)
    mask = (win(g.xyzcc, act)[0] < 0.25).double()

    def lossf(gr, state):
        return ((win(state["B"], act) ** 2).sum(dim=0) * mask).sum()

    La, gGa, gFa, (pa,) = loss_and_grad(g, Gas0, mf0, dt, 6, seg=2, lossf=lossf, params=[g.inflow])
    Lb, gGb, gFb, (pb,) = loss_and_grad_c(g, Gas0, mf0, dt, 6, seg=2, lossf=lossf, params=[g.inflow])
    assert Lb == La, (La, Lb)
    assert _rel((gGb, gFb), (gGa, gFa)) <= 1e-11, _rel((gGb, gFb), (gGa, gFa))
    assert _rel([pb], [pa]) <= 1e-11, (pa, pb)
