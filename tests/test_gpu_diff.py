"""Differentiation form on the GPU: the PyTorch restatement (mage_b200.diffstep)
against the CUDA step through the C ABI.

* forward: the loss after N fixed-dt steps of the CUDA product build equals the
  PyTorch forward on the same device to <= 1e-12 relative;
* gradient: a central finite difference of the CUDA forward along a random
  direction agrees with the reverse-mode gradient to <= 1e-5 relative.
"""
import numpy as np
import pytest
import torch

from mage_b200 import grids
from mage_b200.diffstep import DiffParams, Grid, loss_and_grad, loss_b2, win
from mage_b200.gamera import GameraGPU, GamParams

pytestmark = pytest.mark.gpu


def _cuda_loss(gpu, g, Gx, Fx, dt, nst):
    Nk, Nj, Ni = g.Nk, g.Nj, g.Ni
    with torch.no_grad():
        B = g.bxyz(Fx)
    Gas = np.ascontiguousarray(Gx[:, :Nk, :Nj, :Ni].double().cpu().numpy())
    mf = np.ascontiguousarray(Fx.double().cpu().numpy())
    Bx = np.ascontiguousarray(B[:, :Nk, :Nj, :Ni].double().cpu().numpy())
    gpu.upload_state(Gas, mf, Bx, Gas, mf, 0.0, -dt, dt, 0)
    gpu.step_gamera(nst)
    s = gpu.download_state(old=False)
    Bt = g.cell_box(s["Bxyz"])
    return float(loss_b2(g, {"B": Bt}))


def test_gradient_against_cuda_forward():
    N, dt, nst = (16, 16, 16), 5e-4, 8
    gpu = GameraGPU(GamParams(*N, fixedTimestep=dt))
    gpu.set_geometry(grids.warped_periodic_corners(*N))
    gpu.init_blast_wave()
    st = gpu.download_state(old=False)
    g = Grid(DiffParams(*N), gpu.get_geometry_arrays(), device="cuda")
    rng = np.random.default_rng(11)
    Gas0 = g.cell_box(st["Gas"])
    mf0 = g.face_box(st["magFlux"])
    Gas0 = Gas0 * (1 + 1e-3 * torch.as_tensor(rng.standard_normal(Gas0.shape), device="cuda"))
    mf0 = mf0 + 1e-3 * g.face * torch.as_tensor(rng.standard_normal(mf0.shape), device="cuda")
    L, gG, gF = loss_and_grad(g, Gas0, mf0, dt, nst)
    Lc = _cuda_loss(gpu, g, Gas0, mf0, dt, nst)
    assert abs(Lc - L) <= 1e-12 * abs(L), (Lc, L)
    vG = torch.as_tensor(rng.standard_normal(Gas0.shape), device="cuda") * Gas0.abs()
    vF = torch.as_tensor(rng.standard_normal(mf0.shape), device="cuda")
    eps = 1e-8
    fd = (_cuda_loss(gpu, g, Gas0 + eps * vG, mf0 + eps * vF, dt, nst) -
          _cuda_loss(gpu, g, Gas0 - eps * vG, mf0 - eps * vF, dt, nst)) / (2 * eps)
    ad = float((gG * vG).sum() + (gF * vF).sum())
    assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def _grads(g, Gas0, mf0, dt, nst, cuda_flux, **kw):
    g.cuda_flux = cuda_flux
    return loss_and_grad(g, Gas0, mf0, dt, nst, **kw)


def test_hand_written_flux_adjoint_matches_autograd():
    """The hand-written CUDA adjoints of the flux stage (gam_flux_adjoint) and
    of the electric-field stage (gam_efield_adjoint) inside the reverse sweep
    give the gradient of the pure-autograd sweep to <= 1e-11 relative (L2),
    FP64; their CUDA forwards change the loss by <= 1e-14."""
    N, dt, nst = (16, 16, 16), 5e-4, 4
    gpu = GameraGPU(GamParams(*N))
    gpu.set_geometry(grids.warped_periodic_corners(*N))
    gpu.init_blast_wave()
    st = gpu.download_state(old=False)
    g = Grid(DiffParams(*N), gpu.get_geometry_arrays(), device="cuda")
    rng = np.random.default_rng(3)
    Gas0 = g.cell_box(st["Gas"]) * (1 + 1e-3 * torch.as_tensor(rng.standard_normal((5,) + g.face.shape[1:]), device="cuda"))
    mf0 = g.face_box(st["magFlux"]) + 1e-3 * g.face * torch.as_tensor(rng.standard_normal(g.face.shape), device="cuda")
    La, gGa, gFa = _grads(g, Gas0, mf0, dt, nst, False)
    Lb, gGb, gFb = _grads(g, Gas0, mf0, dt, nst, True)
    assert abs(La - Lb) <= 1e-14 * abs(La)
    num = ((gGa - gGb).norm() ** 2 + (gFa - gFb).norm() ** 2) ** 0.5
    den = (gGa.norm() ** 2 + gFa.norm() ** 2) ** 0.5
    assert float(num / den) <= 1e-11, float(num / den)


def test_hand_written_flux_adjoint_dipole():
    """The same with the background field (dipole in the wind, spherical grid)."""
    from mage_b200 import dipole
    from mage_b200.workloads import DIPOLE_BCS
    N = (16, 8, 8)
    w = dipole.wind_code_units()
    gpu = GameraGPU(GamParams(*N, doBackground=True, bc=DIPOLE_BCS))
    gpu.set_geometry(grids.spherical_corners(*N))
    gpu.set_background_dipole(dipole.M0)
    gpu.init_dipole_wind(w)
    st = gpu.download_state(old=False)
    g = Grid(DiffParams(*N, bc=DIPOLE_BCS), gpu.get_geometry_arrays(), background=gpu.get_background(), wind=w,
             device="cuda")
    dt = 0.5 * st["dt"]
    # the wind start is uniform in v, P and B: exact ties in the limiter, where the
    # two sweeps may pick different (equally valid) subgradients; noise lifts them
    rng = np.random.default_rng(5)
    Gas0 = g.cell_box(st["Gas"]) * (1 + 1e-3 * torch.as_tensor(rng.standard_normal((5,) + g.face.shape[1:]),
                                                               device="cuda"))
    mf0 = g.face_box(st["magFlux"]) + 1e-3 * g.face * torch.as_tensor(rng.standard_normal(g.face.shape), device="cuda")
    act = (4, 4 + N[0] - 1, 4, 4 + N[1] - 1, 4, 4 + N[2] - 1)

    def lossf(gr, state):
        return (win(state["B"], act) ** 2).sum()

    La, gGa, gFa = _grads(g, Gas0, mf0, dt, 3, False, lossf=lossf)
    Lb, gGb, gFb = _grads(g, Gas0, mf0, dt, 3, True, lossf=lossf)
    assert abs(La - Lb) <= 1e-13 * abs(La)
    num = ((gGa - gGb).norm() ** 2 + (gFa - gFb).norm() ** 2) ** 0.5
    den = (gGa.norm() ** 2 + gFa.norm() ** 2) ** 0.5
    assert float(num / den) <= 1e-10, float(num / den)
