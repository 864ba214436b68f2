"""Measurements of the differentiation form (one JSON line).

  python -m mage_b200.diffbench c4            # 64^3 curvilinear blast wave, 20 steps
  python -m mage_b200.diffbench c4_inflow      # the same with an x-inflow / x-outflow
  python -m mage_b200.diffbench c5 --steps 200  # 192x192x256 dipole in the wind
  python -m mage_b200.diffbench cost            # adjoint / forward cost of one step
  python -m mage_b200.diffbench adjstep --n 128 --precisions fp64   # one step's adjoint, 5 calls (profiling)

c4: loss = sum of |B|^2 over the cells centred in [0.6, 0.8]^3 after N fixed-dt
steps from the blast-wave start with seeded Gaussian noise (relative sigma on
rho and P, absolute on v, sigma x face area on the face fluxes); gradient
w.r.t. the start Gas and face fluxes in FP64 and FP32 (checkpoint every
~sqrt(N) steps), and central differences of the CUDA product step and of the
PyTorch forward along a random direction.

c5: the dipole-in-wind set-up on the spherical 192x192x256 grid (background
field, inner sphere, solar wind, zero-gradient axis) with 1e-3 relative noise
on the conserved variables and 1e-3 x face area on the face fluxes; loss = sum of |Bxyz|^2
(the field without the dipole) over active cells with r < 6; FP32 and FP64
gradients with checkpoints every 14 steps and one step's graph at a time.

Both report the time of forward + reverse sweep, peak device memory and the
FP32 gradient's relative L2 distance from the FP64 one.

cost: device time of one step of the product forward (gam_step, the step's
CUDA graph), of the whole-step forward that keeps its intermediates
(gam_step_fwd_save) and of its reverse (gam_step_adj, with the kept
intermediates and with their recomputation), on the blast-wave start at 64^3
(the c4 grid) and 128^3, FP64 and FP32; the adjoint / forward cost is the
reverse's time over the product forward's.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from mage_b200 import dipole, grids
from mage_b200.diffstep import (DiffParams, Grid, KinkCounter, cell_c2p, cell_p2c, count_kinks, loss_and_grad,  # noqa: E501
                               loss_and_grad_c, loss_b2, run, win, G)
from mage_b200.gamera import GameraGPU, GamParams
from mage_b200.workloads import DIPOLE_BCS


def _fortran(g: Grid, Gx, Fx):
    with torch.no_grad():
        B = g.bxyz(Fx)
    Nk, Nj, Ni = g.Nk, g.Nj, g.Ni
    return (np.ascontiguousarray(Gx[:, :Nk, :Nj, :Ni].double().cpu().numpy()),
            np.ascontiguousarray(Fx.double().cpu().numpy()),
            np.ascontiguousarray(B[:, :Nk, :Nj, :Ni].double().cpu().numpy()))


def _rel_l2(a, b):
    num = sum(float((x.double() - y.double()).norm() ** 2) for x, y in zip(a, b))
    den = sum(float(y.double().norm() ** 2) for y in b)
    return (num / den) ** 0.5


def _timed(fn):
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0, torch.cuda.max_memory_allocated() / 1e9


def c4(N=(64, 64, 64), nsteps=20, sigma=1e-3, seed=2024):
    xyz = grids.warped_periodic_corners(*N)
    g0 = GameraGPU(GamParams(*N))
    g0.set_geometry(xyz)
    g0.init_blast_wave()
    st = g0.download_state(old=False)
    dt = 0.5 * st["dt"]
    geo = g0.get_geometry_arrays()
    del g0
    gpu = GameraGPU(GamParams(*N, fixedTimestep=dt))
    gpu.set_geometry(xyz)
    rng = np.random.default_rng(seed)
    g = Grid(DiffParams(*N), geo, device="cuda")
    W = cell_c2p(g.P, list(torch.as_tensor(st["Gas"], device="cuda")))

    def noise(shape):
        return torch.as_tensor(rng.standard_normal(shape), device="cuda")

    sh = W[0].shape
    W = [W[0] * (1 + sigma * noise(sh)), W[1] + sigma * noise(sh), W[2] + sigma * noise(sh), W[3] + sigma * noise(sh),
         W[4] * (1 + sigma * noise(sh))]
    Gas64 = g.cell_box(torch.stack(cell_p2c(g.P, W)))
    mf64 = g.face_box(st["magFlux"]) + sigma * g.face * noise(g.face.shape)
    out = {"config": f"curvilinear blast wave {N[0]}x{N[1]}x{N[2]}, {nsteps} fixed-dt steps (dt = {dt:.4g})",
           "loss": "sum |B|^2 over cells centred in [0.6,0.8]^3", "wrt": "start Gas and face fluxes",
           "impl": "reverse sweep of the step restatement (mage_b200.diffstep): predictor, electric field, fluxes "
                   "and update by hand-written CUDA adjoints (gam_predict_stage, gam_efield_adjoint, gam_flux_adjoint, "
                   "gam_update_stage), boundary gathers and bFlux2Fld by PyTorch autograd; checkpoint every "
                   f"{max(1, int(round(nsteps ** 0.5)))} steps"}
    grads = {}
    for name, dtype in (("fp64", torch.float64), ("fp32", torch.float32)):
        gg = g if dtype == torch.float64 else Grid(DiffParams(*N), geo, dtype=dtype, device="cuda")
        # warm-up with the timed run's own sizes (library, kernels, the allocator's cache of checkpoints)
        loss_and_grad(gg, Gas64.to(dtype), mf64.to(dtype), dt, nsteps)
        (L, gG, gF), el, mem = _timed(lambda: loss_and_grad(gg, Gas64.to(dtype), mf64.to(dtype), dt, nsteps))
        out[name] = {"loss": L, "fwd_plus_adjoint_s": el, "peak_hbm_gb": mem}
        grads[name] = (gG, gF)
    out["fp32_grad_rel_l2_vs_fp64"] = _rel_l2(grads["fp32"], grads["fp64"])
    # the same sweep through the whole-step C entry points (gam_step_fwd_save,
    # gam_step_adj: boundary gathers and bFlux2Fld adjoints on the device too)
    for name, dtype in (("fp64", torch.float64), ("fp32", torch.float32)):
        gg = g if dtype == torch.float64 else Grid(DiffParams(*N), geo, dtype=dtype, device="cuda")
        loss_and_grad_c(gg, Gas64.to(dtype), mf64.to(dtype), dt, nsteps)
        (L, gG, gF), el, mem = _timed(lambda: loss_and_grad_c(gg, Gas64.to(dtype), mf64.to(dtype), dt, nsteps))
        out[name + "_whole_step_c"] = {"loss": L, "fwd_plus_adjoint_s": el, "peak_hbm_gb": mem,
                                       "grad_rel_l2_vs_autograd_sweep": _rel_l2((gG, gF), grads[name])}
    # the same FP64 gradient with the flux stage differentiated by autograd
    # instead of the hand-written CUDA adjoint
    g.cuda_flux = False
    (L, gG, gF), el, mem = _timed(lambda: loss_and_grad(g, Gas64, mf64, dt, nsteps))
    g.cuda_flux = True
    out["fp64_autograd_flux"] = {"fwd_plus_adjoint_s": el, "peak_hbm_gb": mem,
                                 "grad_rel_l2_vs_cuda_flux_adjoint": _rel_l2((gG, gF), grads["fp64"])}
    vG = noise(Gas64.shape) * Gas64.abs()
    vF = noise(mf64.shape)
    ad = float((grads["fp64"][0] * vG).sum() + (grads["fp64"][1] * vF).sum())

    def cuda_loss(Gx, Fx):
        Gas, mf, B = _fortran(g, Gx, Fx)
        gpu.upload_state(Gas, mf, B, Gas, mf, 0.0, -dt, dt, 0)
        gpu.step_gamera(nsteps)
        return float(loss_b2(g, {"B": g.cell_box(gpu.download_state(old=False)["Bxyz"])}))

    def torch_loss(Gx, Fx):
        with torch.no_grad():
            c = {"Gas": Gx, "mf": Fx, "B": g.bxyz(Fx)}
            ce, _ = run(g, c, c, dt, nsteps)
            return float(loss_b2(g, ce))

    # The limiter's kinks (the max/min and sign branches of PDM, the floors)
    # make a central difference approach the reverse mode only as eps -> 0:
    # every decision that switches between the +eps and the -eps run adds a
    # jump term. The PyTorch restatement counts them (KinkCounter) on the same
    # two runs of the PyTorch stages (the torch column). The differentiation
    # form's stated check is a central difference at eps = 1e-6 in FP64.
    fd = {"reverse_mode": ad, "direction": "seeded normal noise x |Gas| on the cells, normal noise on the face fluxes",
          "cuda": {}, "torch": {}, "kinks_crossed": {}}
    for eps in (1e-6, 1e-8, 1e-9, 1e-10, 1e-11):
        d = (cuda_loss(Gas64 + eps * vG, mf64 + eps * vF) - cuda_loss(Gas64 - eps * vG, mf64 - eps * vF)) / (2 * eps)
        fd["cuda"][f"{eps:g}"] = {"central_difference": d, "rel_err": abs(d - ad) / abs(ad)}
        if eps not in (1e-6, 1e-8, 1e-10):
            continue
        k = KinkCounter()
        count_kinks(k)
        g.cuda_flux = False  # every stage as PyTorch expressions, whose branches the counter sees
        try:
            lp = torch_loss(Gas64 + eps * vG, mf64 + eps * vF)
            k.compare()
            lm = torch_loss(Gas64 - eps * vG, mf64 - eps * vF)
        finally:
            count_kinks(None)
            g.cuda_flux = True
        d = (lp - lm) / (2 * eps)
        fd["torch"][f"{eps:g}"] = {"central_difference": d, "rel_err": abs(d - ad) / abs(ad)}
        fd["kinks_crossed"][f"{eps:g}"] = {"switched": k.crossed, "of_decisions": k.decisions}
        del k
        torch.cuda.empty_cache()
    out["fd_check"] = fd
    out["forward_loss_cuda_vs_torch"] = [cuda_loss(Gas64, mf64), torch_loss(Gas64, mf64)]
    return out


INFLOW_BCS = (6, 2, 0, 0, 0, 0)
INFLOW = (1.0, 0.1, 0.5, 0.0, 0.0, 0.5 ** 0.5, 0.5 ** 0.5, 0.3)


def c4_inflow(N=(64, 64, 64), nsteps=20, sigma=1e-3, seed=2024):
    """The c4 grid and start with a uniform inflow on the inner I side
    (rho, P, V, B = INFLOW) and zeroGrad_obcI on the outer one (periodic J, K):
    gradient of sum |B|^2 over the cells centred at x < 0.25 (the part of the
    grid the inflow reaches in the run) w.r.t. the start state and the inflow's
    (rho, P, Vx, Bz), and central differences of the CUDA product step per
    inflow component."""
    xyz = grids.warped_periodic_corners(*N)
    g0 = GameraGPU(GamParams(*N, bc=INFLOW_BCS))
    g0.set_geometry(xyz)
    g0.set_inflow(INFLOW)
    g0.init_blast_wave()
    st = g0.download_state(old=False)
    dt = 0.5 * st["dt"]
    geo = g0.get_geometry_arrays()
    del g0
    gpu = GameraGPU(GamParams(*N, bc=INFLOW_BCS, fixedTimestep=dt))
    gpu.set_geometry(xyz)
    rng = np.random.default_rng(seed)
    P = DiffParams(*N, bc=INFLOW_BCS)
    G64 = st["Gas"] * (1 + sigma * rng.standard_normal(st["Gas"].shape))
    F64 = st["magFlux"] + sigma * np.asarray(geo["face"]) * rng.standard_normal(st["magFlux"].shape)
    names = ("rho", "P", "Vx", "Vy", "Vz", "Bx", "By", "Bz")
    out = {"config": f"curvilinear blast wave {N[0]}x{N[1]}x{N[2]} with a uniform x-inflow "
                     f"{dict(zip(names, INFLOW))} and zero-gradient x-outflow, {nsteps} fixed-dt steps (dt = {dt:.4g})",
           "loss": "sum |B|^2 over cells centred at x < 0.25", "wrt": "start Gas, face fluxes and the inflow state"}
    grads = {}
    for name, dtype in (("fp64", torch.float64), ("fp32", torch.float32)):
        g = Grid(P, geo, dtype=dtype, device="cuda", inflow=INFLOW)
        act = (G, G + N[0] - 1, G, G + N[1] - 1, G, G + N[2] - 1)
        mask = (win(g.xyzcc, act)[0].double() < 0.25).to(dtype)

        def lossf(gr, state):
            return ((win(state["B"], act) ** 2).sum(dim=0) * mask).sum()

        Gas0, mf0 = g.cell_box(G64), g.face_box(F64)
        loss_and_grad(g, Gas0, mf0, dt, nsteps, lossf=lossf, params=[g.inflow])  # warm-up, the timed run's sizes
        (L, gG, gF, (gp,)), el, mem = _timed(lambda: loss_and_grad(g, Gas0, mf0, dt, nsteps, lossf=lossf,
                                                                    params=[g.inflow]))
        out[name] = {"loss": L, "fwd_plus_adjoint_s": el, "peak_hbm_gb": mem,
                     "dloss_dinflow": {names[q]: float(gp[q]) for q in (0, 1, 2, 7)}}
        loss_and_grad_c(g, Gas0, mf0, dt, nsteps, lossf=lossf, params=[g.inflow])  # warm-up
        (Lc, gGc, gFc, (gpc,)), elc, memc = _timed(lambda: loss_and_grad_c(g, Gas0, mf0, dt, nsteps, lossf=lossf,
                                                                          params=[g.inflow]))
        out[name + "_whole_step_c"] = {
            "loss": Lc, "fwd_plus_adjoint_s": elc, "peak_hbm_gb": memc,
            "grad_rel_l2_vs_autograd_sweep": _rel_l2((gGc.cpu(), gFc.cpu()), (gG.cpu(), gF.cpu())),
            "inflow_grad_rel_l2_vs_autograd_sweep": float((gpc - gp).double().norm() / gp.double().norm())}
        grads[name] = gp.double().cpu()
        if name == "fp64":
            lossf64 = lossf
            g64 = g
    out["fp32_inflow_grad_rel_l2_vs_fp64"] = float((grads["fp32"] - grads["fp64"]).norm() / grads["fp64"].norm())
    Gas, mf = np.ascontiguousarray(G64), np.ascontiguousarray(F64)
    with torch.no_grad():
        B = np.ascontiguousarray(g64.bxyz(g64.face_box(F64))[:, :g64.Nk, :g64.Nj, :g64.Ni].cpu().numpy())

    def cuda_loss(w):
        gpu.set_inflow(w)
        gpu.upload_state(Gas, mf, B, Gas, mf, 0.0, -dt, dt, 0)
        gpu.step_gamera(nsteps)
        return float(lossf64(g64, {"B": g64.cell_box(gpu.download_state(old=False)["Bxyz"])}))

    base = np.asarray(INFLOW, dtype=np.float64)
    fd = {}
    for q in (0, 1, 2, 7):
        e = np.zeros(8)
        e[q] = 1e-6 * max(abs(base[q]), 1.0)
        d = (cuda_loss(base + e) - cuda_loss(base - e)) / (2 * e[q])
        ad = out["fp64"]["dloss_dinflow"][names[q]]
        fd[names[q]] = {"central_difference": d, "reverse_mode": ad, "rel_err": abs(d - ad) / abs(ad)}
    out["fd_check_eps_1e-6"] = fd
    return out


def c5(N=(192, 192, 256), nsteps=200, seg=14, precisions=("fp32", "fp64"), seed=2024):
    w = dipole.wind_code_units()
    xyz = grids.spherical_corners(*N)
    gpu = GameraGPU(GamParams(*N, doBackground=True, bc=DIPOLE_BCS))
    gpu.set_geometry(xyz)
    gpu.set_background_dipole(dipole.M0)
    gpu.init_dipole_wind(w)
    st = gpu.download_state(old=False)
    dt = 0.5 * st["dt"]
    geo = gpu.get_geometry_arrays()
    bg = gpu.get_background()
    del gpu
    P = DiffParams(*N, bc=DIPOLE_BCS)
    # noise on the conserved variables and the fluxes: the wind start is
    # uniform in v, P and B, and at exact ties of the limiter the two precisions
    # would pick different (equally valid) subgradients
    rng = np.random.default_rng(seed)
    G64 = st["Gas"] * (1 + 1e-3 * rng.standard_normal(st["Gas"].shape))
    F64 = st["magFlux"] + 1e-3 * np.asarray(geo["face"]) * rng.standard_normal(st["magFlux"].shape)
    out = {"config": f"dipole in a solar wind, spherical {N[0]}x{N[1]}x{N[2]}, {nsteps} fixed-dt steps (dt = {dt:.4g})",
           "loss": "sum |Bxyz|^2 (field without the dipole) over active cells with r < 6",
           "wrt": "start Gas and face fluxes",
           "impl": "reverse sweep of mage_b200.diffstep: predictor, electric field, fluxes, update and the "
                   "inner-sphere / wind fills by hand-written CUDA adjoints, boundary gathers and bFlux2Fld by "
                   f"PyTorch autograd; checkpoint every {seg} steps, one step's graph at a time; *_whole_step_c: "
                   "the same sweep through gam_step_fwd_save_iside / gam_step_adj_iside (no autograd)"}
    grads = {}
    for name in precisions:
        dtype = torch.float64 if name == "fp64" else torch.float32
        g = Grid(P, geo, background=bg, wind=w, dtype=dtype, device="cuda")
        act = (G, G + N[0] - 1, G, G + N[1] - 1, G, G + N[2] - 1)
        xc = win(g.xyzcc, act).double()
        mask = ((xc * xc).sum(dim=0) < 36.0).to(dtype)

        def lossf(gr, state):
            B = win(state["B"], act)
            return ((B * B).sum(dim=0) * mask).sum()

        Gas0, mf0 = g.cell_box(G64).to(dtype), g.face_box(F64)
        loss_and_grad(g, Gas0, mf0, dt, 1, lossf=lossf)  # warm-up
        (L, gG, gF), el, mem = _timed(lambda: loss_and_grad(g, Gas0, mf0, dt, nsteps, seg=seg, lossf=lossf,
                                                             per_step=True))
        out[name] = {"loss": L, "fwd_plus_adjoint_s": el, "s_per_step": el / nsteps, "peak_hbm_gb": mem}
        # the same sweep through the whole-step C entry points (boundary
        # fills, gathers and bFlux2Fld adjoints as kernels, no autograd)
        torch.cuda.empty_cache()
        (Lc, gGc, gFc), elc, memc = _timed(lambda: loss_and_grad_c(g, Gas0, mf0, dt, nsteps, seg=seg, lossf=lossf))
        out[name + "_whole_step_c"] = {"loss": Lc, "fwd_plus_adjoint_s": elc, "s_per_step": elc / nsteps,
                                       "peak_hbm_gb": memc,
                                       "grad_rel_l2_vs_autograd_sweep": _rel_l2((gGc.cpu(), gFc.cpu()),
                                                                                (gG.cpu(), gF.cpu()))}
        grads[name] = (gG.cpu(), gF.cpu())
        del g, Gas0, mf0, gG, gF, gGc, gFc
        torch.cuda.empty_cache()
    if "fp32" in grads and "fp64" in grads:
        out["fp32_grad_rel_l2_vs_fp64"] = _rel_l2(grads["fp32"], grads["fp64"])
    return out


def _ev_ms(fn, reps):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def cost(sizes=((64, 64, 64), (128, 128, 128)), reps=20):
    from mage_b200.diffstep import WholeStep
    from mage_b200.gamera import FP32, FP64
    out = {"what": "device ms per step (CUDA events, after warm-up) on the blast-wave start with a fixed dt; "
                   "adjoint_over_forward = gam_step_adj (saved intermediates) / the product forward step",
           "sizes": {}}
    for N in sizes:
        xyz = grids.warped_periodic_corners(*N)
        g0 = GameraGPU(GamParams(*N))
        g0.set_geometry(xyz)
        g0.init_blast_wave()
        st = g0.download_state(old=False)
        dt = 0.5 * st["dt"]
        geo = g0.get_geometry_arrays()
        del g0
        row = {}
        for name, prec, dtype in (("fp64", FP64, torch.float64), ("fp32", FP32, torch.float32)):
            gpu = GameraGPU(GamParams(*N, fixedTimestep=dt, precision=prec))
            gpu.set_geometry(xyz)
            gpu.init_blast_wave()
            gpu.step_gamera(3)
            gpu.step_gamera(reps)
            fwd = gpu.last_step_ms() / reps
            del gpu
            g = Grid(DiffParams(*N), geo, dtype=dtype, device="cuda")
            G0, F0 = g.cell_box(st["Gas"]), g.face_box(st["magFlux"])
            cur = {"Gas": G0, "mf": F0, "B": g.bxyz(F0)}
            ws = WholeStep(g)
            dn = {"Gas": torch.full_like(G0, 1e-3), "mf": torch.full_like(F0, 1e-3)}
            acc = [torch.zeros_like(G0), torch.zeros_like(F0), torch.zeros_like(G0), torch.zeros_like(F0)]
            ws.forward(cur, cur, dt, dt)
            fsave = _ev_ms(lambda: ws.forward(cur, cur, dt, dt), reps)
            ws.forward(cur, cur, dt, dt)
            adj = _ev_ms(lambda: ws.adjoint(cur, cur, dt, dt, dn, acc, saved=True), reps)
            adj0 = _ev_ms(lambda: ws.adjoint(cur, cur, dt, dt, dn, acc, saved=False), reps)
            row[name] = {"product_forward_ms": fwd, "fwd_save_ms": fsave, "adjoint_ms": adj,
                         "adjoint_with_recompute_ms": adj0, "adjoint_over_forward": adj / fwd}
            del ws, g
            torch.cuda.empty_cache()
        out["sizes"]["x".join(map(str, N))] = row
    return out


def adjstep(n=128, dtype=torch.float64):
    """The whole-step forward and adjoint on the n^3 blast-wave start: two
    forward + adjoint pairs, then three adjoints with the kept intermediates
    (a short, fixed launch sequence for profilers); returns their mean time."""
    from mage_b200.diffstep import WholeStep
    N = (n, n, n)
    g0 = GameraGPU(GamParams(*N))
    g0.set_geometry(grids.warped_periodic_corners(*N))
    g0.init_blast_wave()
    st = g0.download_state(old=False)
    geo = g0.get_geometry_arrays()
    del g0
    g = Grid(DiffParams(*N), geo, dtype=dtype, device="cuda")
    G0, F0 = g.cell_box(st["Gas"]), g.face_box(st["magFlux"])
    cur = {"Gas": G0, "mf": F0, "B": g.bxyz(F0)}
    ws = WholeStep(g)
    dt = 0.5 * st["dt"]
    dn = {"Gas": torch.full_like(G0, 1e-3), "mf": torch.full_like(F0, 1e-3)}
    for _ in range(2):
        ws.forward(cur, cur, dt, dt)
        ws.adjoint(cur, cur, dt, dt, dn, saved=True)
    ms = _ev_ms(lambda: ws.adjoint(cur, cur, dt, dt, dn, saved=True), 2)  # 1 + 2 calls
    return {"grid": list(N), "dtype": str(dtype), "adjoint_ms": ms, "work_gb": ws.work.numel() / 1e9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=["c4", "c4_inflow", "c5", "cost", "adjstep"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--precisions", default="fp32,fp64")
    a = ap.parse_args()
    if a.config == "c4":
        res = c4(nsteps=a.steps or 20)
    elif a.config == "cost":
        res = cost()
    elif a.config == "adjstep":
        res = adjstep(a.n, torch.float32 if a.precisions == "fp32" else torch.float64)
    elif a.config == "c4_inflow":
        res = c4_inflow(nsteps=a.steps or 20)
    else:
        res = c5(nsteps=a.steps or 200, precisions=tuple(a.precisions.split(",")))
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
