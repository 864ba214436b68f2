"""Differentiation form: the PyTorch restatement of the step (mage_b200.diffstep).

* forward: 3 fixed-dt steps of a curvilinear blast wave equal the oracle to
  <= 1e-15 relative (only erfc/exp implementations differ);
* reverse mode: the checkpointed gradient equals the single-segment one
  exactly, and agrees with a central finite difference of the loss along a
  random direction (eps = 1e-8, FP64) to <= 1e-6 relative;
* the kink counter: the limiter decisions that switch between the +eps and
  -eps runs fall with eps (about 3e4, 4e2 and 0 at eps = 1e-5, 1e-7, 1e-9 on
  this case), and once none switches the central difference meets the
  reverse mode to 1e-8.
"""
import numpy as np
import pytest
import torch

from mage_b200 import grids
from mage_b200.diffstep import DiffParams, Grid, KinkCounter, count_kinks, loss_and_grad, loss_b2, run
from oracle.oracle import Oracle, OracleParams
from tests.helpers import GEO_FROM_ORACLE


def _setup(N, dt):
    xyz = grids.warped_periodic_corners(*N)
    o = Oracle(OracleParams(*N, fixedTimestep=True, fixedDT=dt), xyz, "strict")
    o.ic_blast_wave()
    assert o.init_finish() == 0
    g = Grid(DiffParams(*N), {n: o.array(GEO_FROM_ORACLE[n]) for n in GEO_FROM_ORACLE})
    return o, g


def _state(g, o, old=False):
    p = "o" if old else ""
    return {"Gas": g.cell_box(o.array(p + "Gas")), "mf": g.face_box(o.array(p + "magFlux")),
            "B": g.cell_box(o.array(p + "Bxyz"))}


def test_forward_matches_oracle(oracle_built):
    N, dt = (16, 16, 16), 2e-4
    o, g = _setup(N, dt)
    sc = o.scalars()
    cur, old = _state(g, o), _state(g, o, old=True)
    c3, o3 = run(g, cur, old, dt, 3, odt0=sc["time"] - sc["otime"])
    assert o.step(3) == 0
    for name, t, ref in (("Gas", c3["Gas"], o.array("Gas")), ("mf", c3["mf"], o.array("magFlux")),
                         ("B", c3["B"], o.array("Bxyz")), ("oGas", o3["Gas"], o.array("oGas"))):
        a = t.numpy()[:, :ref.shape[1], :ref.shape[2], :ref.shape[3]]
        assert np.abs(a - ref).max() <= 1e-15 * np.abs(ref).max(), name


def test_gradient_checkpointing_and_finite_differences(oracle_built):
    N, dt, nst = (12, 12, 12), 1e-3, 6
    o, g = _setup(N, dt)
    rng = np.random.default_rng(7)
    Gas0 = g.cell_box(o.array("Gas"))
    mf0 = g.face_box(o.array("magFlux"))
    Gas0 = Gas0 * (1 + 1e-3 * torch.as_tensor(rng.standard_normal(Gas0.shape)))
    mf0 = mf0 + 1e-3 * torch.as_tensor(rng.standard_normal(mf0.shape))
    L, gG, gF = loss_and_grad(g, Gas0, mf0, dt, nst)          # segments of ~sqrt(6)
    L1, gG1, gF1 = loss_and_grad(g, Gas0, mf0, dt, nst, seg=nst)
    assert L == L1
    assert torch.equal(gG, gG1) and torch.equal(gF, gF1)

    def Lf(Gx, Fx):
        with torch.no_grad():
            c = {"Gas": Gx, "mf": Fx, "B": g.bxyz(Fx)}
            ce, _ = run(g, c, c, dt, nst)
            return float(loss_b2(g, ce))

    vG = torch.as_tensor(rng.standard_normal(Gas0.shape)) * Gas0.abs()
    vF = torch.as_tensor(rng.standard_normal(mf0.shape))
    eps = 1e-8
    fd = (Lf(Gas0 + eps * vG, mf0 + eps * vF) - Lf(Gas0 - eps * vG, mf0 - eps * vF)) / (2 * eps)
    ad = float((gG * vG).sum() + (gF * vF).sum())
    assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)
    # kinks crossed inside +-eps, and the difference without any
    crossed, errs = [], []
    for eps in (1e-5, 1e-7, 1e-9):  # below ~1e-10 the difference's FP64 cancellation dominates
        k = KinkCounter()
        count_kinks(k)
        try:
            lp = Lf(Gas0 + eps * vG, mf0 + eps * vF)
            k.compare()
            lm = Lf(Gas0 - eps * vG, mf0 - eps * vF)
        finally:
            count_kinks(None)
        crossed.append(k.crossed)
        errs.append(abs((lp - lm) / (2 * eps) - ad) / abs(ad))
        assert k.decisions > 10**6
    assert crossed[0] > crossed[1] > crossed[2], crossed
    assert crossed[-1] == 0, crossed
    for c, e in zip(crossed, errs):
        if c == 0:
            assert e <= 1e-8, (crossed, errs)


def test_per_step_checkpointing_matches(oracle_built):
    N, dt, nst = (12, 12, 12), 1e-3, 5
    o, g = _setup(N, dt)
    Gas0 = g.cell_box(o.array("Gas"))
    mf0 = g.face_box(o.array("magFlux"))
    L, gG, gF = loss_and_grad(g, Gas0, mf0, dt, nst, seg=2)
    L2, gG2, gF2 = loss_and_grad(g, Gas0, mf0, dt, nst, seg=2, per_step=True)
    assert L == L2 and torch.equal(gG, gG2) and torch.equal(gF, gF2)


def test_dipole_wind_forward_matches_oracle(oracle_built):
    """Background field, inner sphere, solar wind and zero-gradient J in the
    PyTorch step: 5 steps equal the oracle to <= 1e-14 relative."""
    from mage_b200 import dipole
    bcs = (3, 4, 2, 2, 0, 0)
    N, dt = (16, 8, 8), 5e-6
    w = dipole.wind_code_units()
    o = Oracle(OracleParams(*N, doBackground=True, M0=dipole.M0, wind=w, bc=bcs, fixedTimestep=True, fixedDT=dt),
               grids.spherical_corners(*N), "strict")
    o.ic_dipole_wind(0.01, 31337)
    assert o.init_finish() == 0
    sc = o.scalars()
    g = Grid(DiffParams(*N, bc=bcs), {n: o.array(GEO_FROM_ORACLE[n]) for n in GEO_FROM_ORACLE},
             background={k: o.array(k) for k in ("fcB0", "bFlux0", "edgB0", "B0", "dpB0")}, wind=w)
    c5, _ = run(g, _state(g, o), _state(g, o, old=True), dt, 5, odt0=sc["time"] - sc["otime"])
    assert o.step(5) == 0
    for name, t, ref in (("Gas", c5["Gas"], o.array("Gas")), ("mf", c5["mf"], o.array("magFlux")),
                         ("B", c5["B"], o.array("Bxyz"))):
        a = t.numpy()[:, :ref.shape[1], :ref.shape[2], :ref.shape[3]]
        assert np.abs(a - ref).max() <= 1e-14 * np.abs(ref).max(), name


INFLOW_BCS = (6, 2, 0, 0, 0, 0)
INFLOW = (1.0, 0.1, 0.5, 0.0, 0.0, 0.5 ** 0.5, 0.5 ** 0.5, 0.3)


def _inflow_setup(N, dt):
    xyz = grids.warped_periodic_corners(*N)
    o = Oracle(OracleParams(*N, fixedTimestep=True, fixedDT=dt, bc=INFLOW_BCS, inflow=INFLOW), xyz, "strict")
    o.ic_blast_wave()
    assert o.init_finish() == 0
    g = Grid(DiffParams(*N, bc=INFLOW_BCS), {n: o.array(GEO_FROM_ORACLE[n]) for n in GEO_FROM_ORACLE}, inflow=INFLOW)
    return o, g


def test_inflow_outflow_forward_matches_oracle(oracle_built):
    """Uniform inflow on the inner I side and zeroGrad_obcI (bcs.F90:820-850)
    on the outer one, periodic J and K: 3 fixed-dt steps equal the oracle to
    <= 1e-15 relative."""
    N, dt = (16, 12, 12), 2e-4
    o, g = _inflow_setup(N, dt)
    sc = o.scalars()
    c3, _ = run(g, _state(g, o), _state(g, o, old=True), dt, 3, odt0=sc["time"] - sc["otime"])
    assert o.step(3) == 0
    for name, t, ref in (("Gas", c3["Gas"], o.array("Gas")), ("mf", c3["mf"], o.array("magFlux")),
                         ("B", c3["B"], o.array("Bxyz"))):
        a = t.numpy()[:, :ref.shape[1], :ref.shape[2], :ref.shape[3]]
        assert np.abs(a - ref).max() <= 1e-15 * np.abs(ref).max(), name


def test_inflow_parameter_gradient(oracle_built):
    """Gradient of sum |B|^2 over the cells with x < 0.3 w.r.t. the inflow
    state (through the boundary fill of every step) against central
    differences of the forward, per component, <= 1e-6 relative; the start
    state's gradient is unchanged by asking for the parameters'."""
    N, dt, nst = (16, 8, 8), 1e-3, 4
    o, g = _inflow_setup(N, dt)
    act = (4, 4 + N[0] - 1, 4, 4 + N[1] - 1, 4, 4 + N[2] - 1)
    from mage_b200.diffstep import win
    mask = (win(g.xyzcc, act)[0] < 0.3).double()

    def lossf(gr, st):
        return ((win(st["B"], act) ** 2).sum(dim=0) * mask).sum()

    Gas0, mf0 = g.cell_box(o.array("Gas")), g.face_box(o.array("magFlux"))
    L, gG, gF, (gp,) = loss_and_grad(g, Gas0, mf0, dt, nst, seg=2, lossf=lossf, params=[g.inflow])
    L1, gG1, gF1 = loss_and_grad(g, Gas0, mf0, dt, nst, seg=2, lossf=lossf)
    assert L == L1 and torch.equal(gG, gG1) and torch.equal(gF, gF1)
    base = g.inflow.clone()

    def Lf(w):
        g.inflow = w
        with torch.no_grad():
            c = {"Gas": Gas0, "mf": mf0, "B": g.bxyz(mf0)}
            ce, _ = run(g, c, c, dt, nst)
            return float(lossf(g, ce))

    for q in (0, 1, 2, 7):  # rho, P, Vx, Bz
        e = torch.zeros(8, dtype=torch.float64)
        e[q] = 1e-6 * max(abs(float(base[q])), 1.0)
        fd = (Lf(base + e) - Lf(base - e)) / (2 * float(e[q]))
        assert abs(fd - float(gp[q])) <= 1e-6 * abs(float(gp[q])), (q, fd, float(gp[q]))
    g.inflow = base
