"""The whole-step entry points of the differentiation form (gam_step_fwd_save,
gam_step_adj: one stepGamera and its adjoint per C call, boundary gathers and
bFlux2Fld on the device) against the PyTorch restatement of the step with its
autograd sweep (mage_b200.diffstep).

* forward: the State after the step equals step() bit for bit (FP64 and FP32,
  periodic and zero-gradient J);
* adjoint: the adjoints of State and oState equal torch.autograd.grad through
  step() to <= 1e-12 relative (L2) in FP64, <= 1e-5 in FP32;
* the checkpointed sweep through the C entry points (loss_and_grad_c) gives
  the loss and gradient of loss_and_grad.
"""
import numpy as np
import pytest
import torch

from mage_b200 import grids
from mage_b200.diffstep import DiffParams, Grid, WholeStep, loss_and_grad, loss_and_grad_c, step
from mage_b200.gamera import GameraGPU, GamParams

pytestmark = pytest.mark.gpu

PERIODIC = (0, 0, 0, 0, 0, 0)
ZEROGRAD_J = (0, 0, 2, 2, 0, 0)
N, DT = (16, 16, 16), 5e-4


def _setup(bc, dtype, seed):
    gpu = GameraGPU(GamParams(*N))
    gpu.set_geometry(grids.warped_periodic_corners(*N))
    gpu.init_blast_wave()
    st = gpu.download_state(old=False)
    geo = gpu.get_geometry_arrays()
    g = Grid(DiffParams(*N, bc=bc), geo, dtype=dtype, device="cuda")
    rng = np.random.default_rng(seed)
    shp = (5,) + tuple(g.face.shape[1:])
    Gas0 = g.cell_box(st["Gas"]) * (1 + 1e-3 * torch.as_tensor(rng.standard_normal(shp), device="cuda").to(dtype))
    mf0 = g.face_box(st["magFlux"]) + 1e-3 * g.face * torch.as_tensor(rng.standard_normal(g.face.shape),
                                                                       device="cuda").to(dtype)
    return g, Gas0, mf0, rng


def _pair(g, Gas0, mf0):
    """(State, oState) one step apart: oState = the start, State = one step on."""
    with torch.no_grad():
        old = {"Gas": Gas0, "mf": mf0, "B": g.bxyz(mf0)}
        cur = step(g, old, old, DT, DT)
    return cur, old


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("bc", [PERIODIC, ZEROGRAD_J], ids=["periodic", "zerogradJ"])
def test_whole_step_forward_equals_restatement(bc, dtype):
    g, Gas0, mf0, _ = _setup(bc, dtype, 5)
    cur, old = _pair(g, Gas0, mf0)
    with torch.no_grad():
        ref = step(g, cur, old, DT, DT)
    out = WholeStep(g).forward(cur, old, DT, DT)
    for k in ("Gas", "mf", "B"):
        assert torch.equal(out[k], ref[k]), (k, float((out[k] - ref[k]).abs().max()))


def _rel(a, b):
    num = sum(float((x - y).norm()) ** 2 for x, y in zip(a, b)) ** 0.5
    den = sum(float(y.norm()) ** 2 for y in b) ** 0.5
    return num / den


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("bc", [PERIODIC, ZEROGRAD_J], ids=["periodic", "zerogradJ"])
def test_whole_step_adjoint_matches_autograd(bc, dtype, tol):
    g, Gas0, mf0, rng = _setup(bc, dtype, 7)
    cur, old = _pair(g, Gas0, mf0)
    leaves = [t.detach().clone().requires_grad_(True) for t in (cur["Gas"], cur["mf"], old["Gas"], old["mf"])]
    with torch.enable_grad():
        c = {"Gas": leaves[0], "mf": leaves[1], "B": g.bxyz(leaves[1])}
        o = {"Gas": leaves[2], "mf": leaves[3], "B": g.bxyz(leaves[3])}
        out = step(g, c, o, DT, DT)
        dn = {k: torch.as_tensor(rng.standard_normal(out[k].shape), device="cuda").to(dtype) for k in out}
        ref = torch.autograd.grad([out[k] for k in ("Gas", "mf", "B")], leaves, [dn[k] for k in ("Gas", "mf", "B")])
    ws = WholeStep(g)
    got = ws.adjoint(cur, old, DT, DT, dn)
    assert _rel(got, ref) <= tol, _rel(got, ref)
    # the intermediates kept by the forward call give the same adjoint, and a
    # second call the same bits (the stencil adjoints are gathered in a fixed
    # order, not added with atomics)
    ws.forward(cur, old, DT, DT)
    got2 = ws.adjoint(cur, old, DT, DT, dn, saved=True)
    for a, b in zip(got2, got):
        assert torch.equal(a, b), float((a - b).abs().max())
    got3 = ws.adjoint(cur, old, DT, DT, dn, saved=True)
    for a, b in zip(got3, got2):
        assert torch.equal(a, b), float((a - b).abs().max())
    # the adjoint reads only what the forward and the adjoint itself wrote: a
    # work area filled with NaN before the forward call gives the same bits
    ws.work.fill_(255)
    ws.forward(cur, old, DT, DT)
    got4 = ws.adjoint(cur, old, DT, DT, dn, saved=True)
    for a, b in zip(got4, got2):
        assert torch.equal(a, b), float((a - b).abs().max())


def test_whole_step_sweep_matches_autograd_sweep():
    g, Gas0, mf0, _ = _setup(PERIODIC, torch.float64, 11)
    La, gGa, gFa = loss_and_grad(g, Gas0, mf0, DT, 6, seg=2)
    Lb, gGb, gFb = loss_and_grad_c(g, Gas0, mf0, DT, 6, seg=2)
    assert Lb == La, (La, Lb)
    assert _rel((gGb, gFb), (gGa, gFa)) <= 1e-11, _rel((gGb, gFb), (gGa, gFa))

