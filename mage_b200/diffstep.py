"""Differentiable stepGamera in PyTorch operations (FP64 or FP32, CPU or GPU).

The same step as the CUDA kernels of ``csrc/gam_step_impl.cuh`` (periodic
boundaries, no background field, 8CENT or 7UP reconstruction, LFM limiter,
fixed dt), written as whole-array tensor expressions so that autograd gives its
reverse mode. It is the gradient reference of the differentiation form and its
first implementation: ``loss_and_grad`` runs N steps with sqrt(N)-style
checkpointing (segments are recomputed during the reverse sweep).

Arrays use the padded-box convention of the CUDA code without padding: every
field is a tensor ``(nc, Nk+1, Nj+1, Ni+1)`` indexed ``[c, kk, jj, ii]`` with box
index ``ii = i - isg`` (Ni = Nip + 8); cell fields leave the last slot of each
axis unused. Routines and their reference (file:line):

  predictor        Predictor / PredictCell / ExtrapAB2   mhdgroup.F90:444-615,709-717
  mom2face, vxb    CalcElecField / Mom2Face / EdgeLRs     fields.F90:70-517
  stress           Fluxes / GasKinFlux / MagKinFlux       stress.F90:204-599
  recon            Cen8LRs / Up7LRs / pdmLR / PDM         recon.F90:125-301
  update           applyUpdate / E2Flux / CellMaxwell     mhdgroup.F90:79-329, fields.F90:18-51
  bcs              EnforceBCs (periodic) + bFlux2Fld      step.F90:17-55, bcs.F90:279-450
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

G = 4
TINY = 1.0e-12
PI = 3.141592653589793
W8 = (-3.0 / 840.0, 29.0 / 840.0, -139.0 / 840.0, 533.0 / 840.0, 533.0 / 840.0, -139.0 / 840.0, 29.0 / 840.0,
      -3.0 / 840.0)
UP7 = (-3.0 / 420.0, 25.0 / 420.0, -101.0 / 420.0, 319.0 / 420.0, 214.0 / 420.0, -38.0 / 420.0, 4.0 / 420.0)


@dataclass
class DiffParams:
    Nip: int
    Njp: int
    Nkp: int
    gamma: float = 5.0 / 3.0
    CFL: float = 0.3
    pdmb: float = 0.75
    Vd0: float = 0.5
    cHogH: float = 0.25
    dFloor: float = 1.0e-12
    pFloor: float = 1.0e-12
    up7: bool = False
    # boundary kinds per side (INI, OUTI, INJ, OUTJ, INK, OUTK): 0 periodic,
    # 1 none, 2 zero-gradient (J, outer I), 3 inner sphere (inner I), 4 solar
    # wind (outer I), 6 uniform inflow (inner I)
    bc: tuple = (0, 0, 0, 0, 0, 0)


# ----------------------------------------------------------------- kinks
class KinkCounter:
    """Counts the non-smooth decisions (max/min operands, signs, |x| and the
    sqrt at 0, the limiter's branches) that differ between two evaluations of
    the PyTorch step: "record" stores every decision of the first run in
    order, "compare" walks the second run's decisions against them and counts
    the elements that switched (kinks crossed between the two inputs)."""

    def __init__(self):
        self.mode, self.masks, self.pos, self.crossed, self.decisions = "record", [], 0, 0, 0

    def see(self, m):
        if self.mode == "record":
            self.masks.append(m.detach().clone())
            self.decisions += m.numel()
        else:
            self.crossed += int((self.masks[self.pos] != m.detach()).sum())
            self.pos += 1

    def compare(self):
        self.mode, self.pos, self.crossed = "compare", 0, 0


_KINKS: KinkCounter | None = None


def count_kinks(counter: KinkCounter | None):
    """Install (or remove, with None) the counter the branch helpers report to."""
    global _KINKS
    _KINKS = counter


def _see(m):
    if _KINKS is not None:
        _KINKS.see(m)
    return m


# ----------------------------------------------------------------- helpers
def rmax(a, b):
    """std::max: (a < b) ? b : a."""
    return torch.where(_see(a < b), b, a)


def rmin(a, b):
    """std::min: (b < a) ? b : a."""
    return torch.where(_see(b < a), b, a)


def kabs(x):
    """|x|, its kink at 0 reported to the kink counter."""
    _see(x < 0)
    return torch.abs(x)


def ksign(x):
    """copysign(1, x), its switch at 0 reported to the kink counter."""
    one = torch.ones_like(x)
    _see(torch.signbit(x))
    return torch.copysign(one, x)


def safe_sqrt(x):
    """sqrt with a zero (sub)gradient at 0 instead of inf * 0."""
    pos = _see(x > 0)
    return torch.where(pos, torch.sqrt(torch.where(pos, x, torch.ones_like(x))), torch.zeros_like(x))


def win(a, rng, off=(0, 0, 0)):
    """a[..., k, j, i] over the inclusive box range rng = (i0, i1, j0, j1, k0, k1)
    shifted by off = (di, dj, dk)."""
    i0, i1, j0, j1, k0, k1 = rng
    di, dj, dk = off
    return a[..., k0 + dk:k1 + dk + 1, j0 + dj:j1 + dj + 1, i0 + di:i1 + di + 1]


def unit(d, n):
    o = [0, 0, 0]
    o[d] = n
    return tuple(o)


def add(o1, o2):
    return (o1[0] + o2[0], o1[1] + o2[1], o1[2] + o2[2])


def put(base, rng, val):
    """Copy of base with val written over the box range rng (autograd-safe)."""
    out = base.clone()
    i0, i1, j0, j1, k0, k1 = rng
    out[..., k0:k1 + 1, j0:j1 + 1, i0:i1 + 1] = val
    return out


def central8(q):
    s = torch.zeros_like(q[0])
    for n in range(8):
        s = s + W8[n] * q[n]
    return s


def pdm_lr(pdmb, v, Qi):
    """pdmLR (recon.F90:231-272) on the 4-point limiter stencil v[0..3]."""
    v0, v1, v2, v3 = v
    maxV, minV = rmax(v1, v2), rmin(v1, v2)
    vN = rmax(minV, rmin(Qi, maxV))
    dv0, dv1, dv2 = pdmb * (v1 - v0), pdmb * (v2 - v1), pdmb * (v3 - v2)
    s0, s1, s2 = ksign(dv0), ksign(dv1), ksign(dv2)
    q0, q1 = torch.abs(s0 + s1), torch.abs(s1 + s2)
    dvL, dvR = vN - v1, v2 - vN
    zero = torch.zeros_like(vN)
    Ql = vN - s1 * rmax(zero, kabs(dvL) - q0 * kabs(dv0))
    Qr = vN + s1 * rmax(zero, kabs(dvR) - q1 * kabs(dv2))
    return Ql, Qr


def pdm1(pdmb, q0, q1, q2, qI):
    """PDM (recon.F90:275-301)."""
    maxQ, minQ = rmax(q1, q2), rmin(q1, q2)
    qN = rmax(minQ, rmin(qI, maxQ))
    dq0, dq1 = pdmb * (q1 - q0), pdmb * (q2 - q1)
    s0, s1 = ksign(dq0), ksign(dq1)
    s01 = torch.abs(s0 + s1)
    dqL = qN - q1
    return qN - s1 * rmax(torch.zeros_like(qN), kabs(dqL) - s01 * kabs(dq0))


def lrs_from_qdv(P: DiffParams, qdv, nq, Vi):
    """Cen8LRs / Up7LRs on the volume-weighted stencil qdv[0..7] (cells -4..3),
    limited by PDM on nq[0..3] (cells -2..1)."""
    if not P.up7:
        Qi = central8(qdv) / Vi
        return pdm_lr(P.pdmb, nq, Qi)
    a = qdv[0] * UP7[0]
    for n in range(1, 7):
        a = a + qdv[n] * UP7[n]
    b = qdv[7] * UP7[0]
    for n in range(1, 7):
        b = b + qdv[7 - n] * UP7[n]
    Ql, Qr = a / Vi, b / Vi
    return pdm1(P.pdmb, nq[0], nq[1], nq[2], Ql), pdm1(P.pdmb, nq[3], nq[2], nq[1], Qr)


def cell_c2p(P, U):
    rho = U[0]
    Vx, Vy, Vz = U[1] / rho, U[2] / rho, U[3] / rho
    KinE = 0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz)
    return [rmax(rho, torch.full_like(rho, P.dFloor)), Vx, Vy, Vz,
            rmax((P.gamma - 1) * (U[4] - KinE), torch.full_like(rho, P.pFloor))]


def cell_p2c(P, W):
    rho = rmax(W[0], torch.full_like(W[0], P.dFloor))
    Vx, Vy, Vz = W[1], W[2], W[3]
    IntE = rmax(W[4], torch.full_like(W[4], P.pFloor)) / (P.gamma - 1)
    KinE = 0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz)
    return [rho, rho * Vx, rho * Vy, rho * Vz, IntE + KinE]


def block_c2p(P, U):
    D = rmax(U[0], torch.full_like(U[0], P.dFloor))
    Mx, My, Mz = U[1], U[2], U[3]
    KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D
    Pr = rmax((P.gamma - 1) * (U[4] - KinE), torch.full_like(D, P.pFloor))
    return [D, Mx / D, My / D, Mz / D, Pr]


# ----------------------------------------------------------------- grid
def _gather_adjoint_plan(src: torch.Tensor):
    """Static plan for the adjoint of out[j] = x[src[j]] (the boundary
    gather): positions that are their own source keep their adjoint, every
    other position's adjoint is added to its source. The sources that receive
    are grouped with their (at most K) destinations in a padded table, so the
    reverse sum runs as K gathers in a fixed order (deterministic, unlike an
    atomic scatter)."""
    s = src.cpu().numpy()
    n = s.size
    j = np.arange(n)
    self_src = s == j
    gj = j[~self_src]
    gs = s[~self_src]
    order = np.argsort(gs, kind="stable")
    gj, gs = gj[order], gs[order]
    uniq, start, counts = np.unique(gs, return_index=True, return_counts=True)
    K = int(counts.max()) if counts.size else 0
    table = np.full((uniq.size, max(K, 1)), n, dtype=np.int64)  # n: a zero slot appended in backward
    for k in range(K):
        has = counts > k
        table[has, k] = gj[start[has] + k]
    dev = src.device
    return {"keep": torch.as_tensor(self_src, device=dev), "recv": torch.as_tensor(uniq, device=dev),
            "table": torch.as_tensor(table, device=dev), "K": K}


class _GatherFn(torch.autograd.Function):
    """x[:, src] with the deterministic reverse of _gather_adjoint_plan."""

    @staticmethod
    def forward(ctx, x, src, plan):
        ctx.plan = plan
        return x[:, src]

    @staticmethod
    def backward(ctx, g):
        p = ctx.plan
        gx = g * p["keep"].to(g.dtype)
        if p["K"]:
            gz = torch.cat([g, torch.zeros_like(g[:, :1])], dim=1)
            acc = gz[:, p["table"][:, 0]]
            for k in range(1, p["K"]):
                acc = acc + gz[:, p["table"][:, k]]
            gx[:, p["recv"]] += acc
        return gx, None, None


class Grid:
    """Metric tensors in the unpadded box convention (from the C ABI's
    Fortran-layout geometry arrays)."""

    def __init__(self, P: DiffParams, geo: dict, background: dict | None = None, wind=None, dtype=torch.float64,
                 device="cpu", inflow=None):
        self.P = P
        self.Ni, self.Nj, self.Nk = P.Nip + 2 * G, P.Njp + 2 * G, P.Nkp + 2 * G
        self.dtype, self.device = dtype, device

        def face(a):
            return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=device)

        def cell(a):
            a = np.asarray(a)
            out = np.zeros((a.shape[0], self.Nk + 1, self.Nj + 1, self.Ni + 1))
            out[:, :self.Nk, :self.Nj, :self.Ni] = a
            return torch.as_tensor(out, dtype=dtype, device=device)

        self.face = face(geo["face"])
        self.xfc = face(geo["xfc"])
        self.Tf = face(geo["Tf"])
        self.edge = face(geo["edge"])
        self.Te = face(geo["Te"])
        self.Teb = face(geo["Teb"])
        self.vol = cell(geo["volume"])[0]
        self.xyzcc = cell(geo["xyzcc"])
        # face centroid - cell centroid of the six faces of each cell (FP64,
        # rounded once): the FP32 form's bFlux2Fld operand, as in the CUDA form
        xf = np.ascontiguousarray(geo["xfc"], dtype=np.float64)
        xc = np.zeros((3,) + xf.shape[1:])
        xc[:, :self.Nk, :self.Nj, :self.Ni] = np.asarray(geo["xyzcc"])
        off = np.zeros((18,) + xf.shape[1:])
        for d in range(3):
            up = [0, 0, 0]
            up[2 - d] = 1
            for x in range(3):
                off[x + 3 * (2 * d)] = xf[x + 3 * d] - xc[x]
                shifted = np.zeros_like(xf[x + 3 * d])
                sl_dst = tuple(slice(0, n - u) for n, u in zip(shifted.shape, up))
                sl_src = tuple(slice(u, n) for n, u in zip(shifted.shape, up))
                shifted[sl_dst] = xf[x + 3 * d][sl_src]
                off[x + 3 * (2 * d + 1)] = shifted - xc[x]
        self.dxf = torch.as_tensor(off, dtype=dtype, device=device)
        # background field (AddB0 arrays, cell-sized; kept in FP64 like the CUDA forms)
        self.bg = None
        if background is not None:
            self.bg = {k: torch.as_tensor(self._cellpad(background[k]), dtype=torch.float64, device=device)
                       for k in ("fcB0", "bFlux0", "edgB0", "B0", "dpB0")}
        # the flux stage and its adjoint as hand-written CUDA kernels (on CUDA
        # tensors, 8CENT); False: the PyTorch expressions and autograd
        self.cuda_flux = torch.device(device).type == "cuda" and not P.up7
        # the inflow state {rho, P, Vx, Vy, Vz, Bx, By, Bz} of bc[0] = 6: a
        # tensor, so that a caller may ask for gradients with respect to it
        self.inflow = None
        if P.bc[0] == 6:
            assert inflow is not None, "the inflow boundary needs its state"
            self.inflow = torch.as_tensor(inflow, dtype=dtype, device=device)
        self.wind = None
        if P.bc[1] == 4:
            assert wind is not None, "the solar-wind boundary needs the wind state"
            self.wind = self._wind_tables(geo, np.asarray(wind, dtype=np.float64))
        self._bc_maps()

    def _cellpad(self, a):
        a = np.asarray(a)
        out = np.zeros((a.shape[0], self.Nk + 1, self.Nj + 1, self.Ni + 1))
        out[:, :self.Nk, :self.Nj, :self.Ni] = a
        return out

    def _wind_tables(self, geo, w):
        """Blend weights (wgtWind, apps/wind.F90:180-203; RampDown, math.F90:97-111)
        and wind face fluxes of the 4 outer-I ghost layers, as gam_set_wind
        computes them: cell weight at ig = ie+n, I-face weight/flux at ig+1,
        J- and K-face weights/fluxes at ig, for every (j, k) of the face box."""
        P = self.P
        i0 = G + P.Nip
        V, Bsw = w[2:5], w[5:8]

        def norm_vec(a):
            nA = np.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
            safe = np.where(nA <= 1e-12, 1.0, nA)
            return np.where(nA <= 1e-12, 0.0, a / safe)

        def wgt(x):
            nH = norm_vec(x)
            vH = norm_vec(V.reshape(3, *([1] * (x.ndim - 1))))
            dTh = np.arccos(-vH[0] * nH[0] + -vH[1] * nH[1] + -vH[2] * nH[2]) * 180.0 / PI
            rScl = (dTh - 90.0) / 90.0
            with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                ramp = np.exp(-1.0 / (1.0 - rScl * rScl) + 1.0)
            return np.where(dTh <= 90.0, 1.0, np.where(dTh >= 180.0, 0.0, ramp))

        xcc = np.asarray(geo["xyzcc"])[:, :, :, i0:i0 + 4]          # (3, Nk, Nj, 4)
        xfc = np.asarray(geo["xfc"])
        Tf = np.asarray(geo["Tf"])
        face = np.asarray(geo["face"])
        t = {"wC": wgt(xcc)}
        for d in range(3):
            sl = slice(i0 + 1, i0 + 5) if d == 0 else slice(i0, i0 + 4)
            xf = xfc[3 * d:3 * d + 3, :, :, sl]
            nH = Tf[9 * d:9 * d + 3, :, :, sl]
            t[f"wF{d}"] = wgt(xf)
            t[f"sF{d}"] = face[d, :, :, sl] * (nH[0] * Bsw[0] + nH[1] * Bsw[1] + nH[2] * Bsw[2])
        out = {k: torch.as_tensor(v, dtype=self.dtype, device=self.device) for k, v in t.items()}
        out["state"] = w
        return out

    def cell_box(self, a):
        """Fortran-layout cell array (nc, Nk, Nj, Ni) -> box tensor."""
        a = a if torch.is_tensor(a) else torch.as_tensor(np.asarray(a))
        a = a.to(dtype=self.dtype, device=self.device)
        out = torch.zeros((a.shape[0], self.Nk + 1, self.Nj + 1, self.Ni + 1), dtype=self.dtype, device=self.device)
        out[:, :self.Nk, :self.Nj, :self.Ni] = a
        return out

    def face_box(self, a):
        a = a if torch.is_tensor(a) else torch.as_tensor(np.ascontiguousarray(a))
        return a.to(dtype=self.dtype, device=self.device)

    def _bc_maps(self):
        """Flat gather indices of the boundary conditions that copy values
        (periodic bcs.F90:279-450, zero-gradient J :853-892), composed in the
        reference's order: the value at (i, j, k) comes from the I map of the J
        map of the K map of its index; the zero-gradient J map applies over the
        cell ranges of i and k only. SphIn and the wind are applied in place
        before the gather (step())."""
        P = self.P
        nx, ny, nz = self.Ni + 1, self.Nj + 1, self.Nk + 1
        n = (P.Nip, P.Njp, P.Nkp)
        bc = P.bc

        def lo(kind, x, nn):
            x = x.copy()
            m = x < G
            if kind == 0:
                x[m] = x[m] + nn
            elif kind == 2:
                x[m] = G
            return x

        def hi(kind, x, nn, normal):
            x = x.copy()
            m = ((x >= G + nn + 1) & (x <= G + nn + 4)) if normal else ((x >= G + nn) & (x <= G + nn + 3))
            if kind == 0:
                x[m] = x[m] - nn
            elif kind == 2:
                x[m] = (G + nn) if normal else (G + nn - 1)
            return x

        kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        self.bc_src = {}
        for comp in (-1, 0, 1, 2):
            sk = kk
            if bc[4] == 0:
                sk = hi(0, lo(0, sk, n[2]), n[2], comp == 2)
            sjm = hi(bc[3], lo(bc[2], jj, n[1]), n[1], comp == 1)
            cond = np.ones_like(ii, dtype=bool) if bc[2] == 0 else ((ii < self.Ni) & (sk < self.Nk))
            sj = np.where(cond, sjm, jj)
            si = ii
            if bc[0] == 0:
                si = hi(0, lo(0, si, n[0]), n[0], comp == 0)
            src = (sk * ny + sj) * nx + si
            if comp == -1:  # cell values: the cell box only
                keep = (ii >= self.Ni) | (jj >= self.Nj) | (kk >= self.Nk)
                src = np.where(keep, (kk * ny + jj) * nx + ii, src)
            self.bc_src[comp] = torch.as_tensor(src.reshape(-1), device=self.device)
        self.bc_adj = {c: _gather_adjoint_plan(self.bc_src[c]) for c in self.bc_src}

    def bxyz(self, mf):
        """gamCellBxyz (gridutils.F90:648-680) on every cell of the box."""
        rc = (0, self.Ni - 1, 0, self.Nj - 1, 0, self.Nk - 1)
        fI, fIp = win(mf[0], rc), win(mf[0], rc, (1, 0, 0))
        fJ, fJp = win(mf[1], rc), win(mf[1], rc, (0, 1, 0))
        fK, fKp = win(mf[2], rc), win(mf[2], rc, (0, 0, 1))
        dV = win(self.vol, rc)
        if self.dtype == torch.float32:
            d = self.dxf
            B = [(fIp * win(d[x + 3], rc) + fJp * win(d[x + 9], rc) + fKp * win(d[x + 15], rc) - fI * win(d[x], rc) -
                  fJ * win(d[x + 6], rc) - fK * win(d[x + 12], rc)) / dV for x in range(3)]
            return put(torch.zeros_like(mf), rc, torch.stack(B))
        Div = fIp - fI + fJp - fJ + fKp - fK
        B = []
        for x in range(3):
            t = (fIp * win(self.xfc[x], rc, (1, 0, 0)) + fJp * win(self.xfc[x + 3], rc, (0, 1, 0)) +
                 fKp * win(self.xfc[x + 6], rc, (0, 0, 1)) - fI * win(self.xfc[x], rc) -
                 fJ * win(self.xfc[x + 3], rc) - fK * win(self.xfc[x + 6], rc)) / dV
            B.append(t - Div * win(self.xyzcc[x], rc) / dV)
        return put(torch.zeros_like(mf), rc, torch.stack(B))


# ----------------------------------------------------------------- the step
def _predict_torch(g: Grid, cur: dict, old: dict, pdt: float, odt: float):
    """Predictor (mhdgroup.F90:444-615) as tensor expressions."""
    P = g.P
    Ni, Nj, Nk = g.Ni, g.Nj, g.Nk
    allc = (0, Ni - 1, 0, Nj - 1, 0, Nk - 1)
    Q, oQ = cur["mf"], old["mf"]
    hm = Q + pdt * ((Q - oQ) / odt)
    A = g.face
    Am = rmax(A, torch.full_like(A, TINY))
    bh = hm / Am
    abh = A * bh
    Bnf = hm / A
    bn = Q / Am
    Uc = [win(cur["Gas"][v], allc) for v in range(5)]
    Uo = [win(old["Gas"][v], allc) for v in range(5)]
    W, oW = cell_c2p(P, Uc), cell_c2p(P, Uo)
    pW = [W[v] + pdt * ((W[v] - oW[v]) / odt) for v in range(5)]
    pW[0] = rmax(pW[0], torch.full_like(pW[0], P.dFloor))
    pW[4] = rmax(pW[4], torch.full_like(pW[4], P.pFloor))
    pQ = cell_p2c(P, pW)
    Wh = block_c2p(P, pQ)
    Wn = block_c2p(P, Uc)
    vol = win(g.vol, allc)
    zeros5 = torch.zeros_like(cur["Gas"])
    QW = put(zeros5, allc, torch.stack([vol * Wh[v] for v in range(5)]))
    WnB = put(zeros5, allc, torch.stack(Wn))
    Dh = put(torch.zeros_like(g.vol), allc, Wh[0])
    Dm = rmax(pQ[0], torch.full_like(pQ[0], P.dFloor))
    VdV = put(torch.zeros_like(cur["B"]), allc, torch.stack([vol * pQ[1 + x] / Dm for x in range(3)]))
    QB = g.bxyz(hm) * g.vol
    return QW, WnB, Dh, VdV, QB, abh, Bnf, bn


def _update_torch(g: Grid, cur: dict, E, gF, mF, dt: float):
    """applyUpdate: E2Flux, CellReynolds, CellMaxwell (mhdgroup.F90:79-329) as tensor expressions."""
    P = g.P
    gm1 = P.gamma - 1
    Np = (P.Nip, P.Njp, P.Nkp)
    inr = (G, G + Np[0], G, G + Np[1], G, G + Np[2])
    dfi = win(E[2], inr, (0, 1, 0)) - win(E[2], inr) - win(E[1], inr, (0, 0, 1)) + win(E[1], inr)
    dfj = win(E[0], inr, (0, 0, 1)) - win(E[0], inr) - win(E[2], inr, (1, 0, 0)) + win(E[2], inr)
    dfk = win(E[1], inr, (1, 0, 0)) - win(E[1], inr) - win(E[0], inr, (0, 1, 0)) + win(E[0], inr)
    mfn = put(cur["mf"], inr, torch.stack([win(cur["mf"][0], inr) - dt * dfi, win(cur["mf"][1], inr) - dt * dfj,
                                          win(cur["mf"][2], inr) - dt * dfk]))
    act = (G, G + Np[0] - 1, G, G + Np[1] - 1, G, G + Np[2] - 1)
    dV = win(g.vol, act)
    U = []
    for v in range(5):
        dGasH = (win(gF[0][v], act) - win(gF[0][v], act, (1, 0, 0)) + win(gF[1][v], act) -
                 win(gF[1][v], act, (0, 1, 0)) + win(gF[2][v], act) - win(gF[2][v], act, (0, 0, 1))) / dV
        U.append(win(cur["Gas"][v], act) + dt * dGasH)
    dGasM = [(win(mF[0][x], act) - win(mF[0][x], act, (1, 0, 0)) + win(mF[1][x], act) - win(mF[1][x], act, (0, 1, 0)) +
              win(mF[2][x], act) - win(mF[2][x], act, (0, 0, 1))) / dV for x in range(3)]
    if g.bg is not None:
        dGasM = [dGasM[x] + win(g.bg["dpB0"][x], act).to(dV.dtype) for x in range(3)]
    # CellMaxwell (mhdgroup.F90:299-329)
    Dn = rmax(U[0], torch.full_like(U[0], P.dFloor))
    Mx, My, Mz, TotE = U[1], U[2], U[3], U[4]
    KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / Dn
    Pr = rmax(gm1 * (TotE - KinE), torch.full_like(Dn, P.pFloor))
    Mx, My, Mz = Mx + dt * dGasM[0], My + dt * dGasM[1], Mz + dt * dGasM[2]
    KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / Dn
    Gas = put(cur["Gas"], act, torch.stack([Dn, Mx, My, Mz, KinE + Pr / gm1]))
    return Gas, mfn


def step(g: Grid, cur: dict, old: dict, dt: float, odt: float):
    """One stepGamera with a fixed dt. cur/old: {"Gas": (5,...), "mf": (3,...),
    "B": (3,...)} box tensors of State (n) and oState (n-1); odt = time - otime
    after the AdvanceMHD time trap. Returns State (n+1) (boundaries filled)."""
    P = g.P
    Ni, Nj, Nk = g.Ni, g.Nj, g.Nk
    pdt = 0.5 * dt
    gm1 = P.gamma - 1
    allf = (0, Ni, 0, Nj, 0, Nk)
    allc = (0, Ni - 1, 0, Nj - 1, 0, Nk - 1)

    # --- Predictor (every face and cell of the box)
    A = g.face
    if g.cuda_flux:
        QW, WnB, Dh, VdV, QB, abh, Bnf, bn = _PredictFn.apply(cur["Gas"], cur["mf"], old["Gas"], old["mf"], g, pdt, odt)
    else:
        QW, WnB, Dh, VdV, QB, abh, Bnf, bn = _predict_torch(g, cur, old, pdt, odt)
    Blim = cur["B"]

    # --- CalcElecField
    Np = (P.Nip, P.Njp, P.Nkp)
    mf_r = [(0, Ni - 1, G, G + Np[1], 0, Nk - 1), (0, Ni - 1, 0, Nj - 1, G, G + Np[2]), (G, G + Np[0], 0, Nj - 1, 0, Nk - 1)]
    ed_r = [(G, G + Np[0] - 1, G, G + Np[1], G, G + Np[2]), (G, G + Np[0], G, G + Np[1] - 1, G, G + Np[2]),
            (G, G + Np[0], G, G + Np[1], G, G + Np[2] - 1)]
    E = []
    if g.cuda_flux:
        Ea = _EFieldFn.apply(Dh, abh, bn, VdV, g, dt)
        E = [Ea[0], Ea[1], Ea[2]]
    for eD in ([] if g.cuda_flux else range(3)):
        dT1, dT2 = (eD + 1) % 3, (eD + 2) % 3
        r = mf_r[eD]
        dV = rmax(central8([win(g.vol, r, unit(dT1, n - 4)) for n in range(8)]), torch.full_like(win(g.vol, r), TINY))
        Af = win(A[dT1], r)
        AVf = torch.zeros_like(cur["B"])
        AVf = put(AVf, r, torch.stack([Af * (central8([win(VdV[x], r, unit(dT1, n - 4)) for n in range(8)]) / dV)
                                       for x in range(3)]))
        r = ed_r[eD]
        e1 = 1 if eD == 0 else 0
        e2 = 1 if eD == 2 else 2
        o1, o2 = unit(e1, -1), unit(e2, -1)
        Dc = 0.25 * (win(Dh, r) + win(Dh, r, o1) + win(Dh, r, o2) + win(Dh, r, add(o1, o2)))

        def edge_lrs(a, bd):
            area = [win(A[a], r, unit(bd, n - 4)) for n in range(8)]
            qdv = [win(abh[a], r, unit(bd, n - 4)) for n in range(8)]
            nmag = [win(bn[a], r, unit(bd, m - 2)) for m in range(4)]
            Vi = central8(area)
            bL, bR = lrs_from_qdv(P, qdv, nmag, Vi)
            return bL * Vi, bR * Vi, Vi

        bT1L, bT1R, fA1 = edge_lrs(dT1, dT2)
        bT2L, bT2R, fA2 = edge_lrs(dT2, dT1)
        dA = rmax(fA1, torch.full_like(fA1, TINY))
        VC = [central8([win(AVf[x], r, unit(dT2, n - 4)) for n in range(8)]) / dA for x in range(3)]
        Te = [win(g.Te[q + 9 * eD], r) for q in range(9)]
        v1 = VC[0] * Te[3] + VC[1] * Te[4] + VC[2] * Te[5]
        v2 = VC[0] * Te[6] + VC[1] * Te[7] + VC[2] * Te[8]
        vDiff = safe_sqrt(v1 * v1 + v2 * v2)
        xni, yni, xnj, ynj = (win(g.Teb[q + 4 * eD], r) for q in range(4))
        detT = 1.0 / (xni * ynj - xnj * yni)
        bT1 = 0.5 * (bT1L + bT1R) / fA1
        bT2 = 0.5 * (bT2L + bT2R) / fA2
        db1 = (bT1R - bT1L) / fA1
        db2 = (bT2R - bT2L) / fA2
        Jd = db2 - db1
        b1 = detT * (ynj * bT1 - yni * bT2)
        b2 = detT * (-(xnj * bT1) + xni * bT2)
        if g.bg is not None:
            b1 = b1 + win(g.bg["edgB0"][0 + 2 * eD], r).to(b1.dtype)
            b2 = b2 + win(g.bg["edgB0"][1 + 2 * eD], r).to(b2.dtype)
        vA = safe_sqrt(b1 * b1 + b2 * b2) / torch.sqrt(Dc)
        vDiff = vDiff + vA
        edge = win(g.edge[eD], r)
        vDiff = rmin(vDiff, P.CFL * edge / dt)
        e = -(v1 * b2 - v2 * b1) + P.Vd0 * vDiff * Jd
        E.append(put(torch.zeros_like(g.vol), r, e * edge))

    # --- CalcStress
    zeros5 = torch.zeros_like(cur["Gas"])
    fr = [(G, G + Np[0], G, G + Np[1] - 1, G, G + Np[2] - 1), (G, G + Np[0] - 1, G, G + Np[1], G, G + Np[2] - 1),
          (G, G + Np[0] - 1, G, G + Np[1] - 1, G, G + Np[2])]
    gF, mF = [], []
    if g.cuda_flux:
        gFa, mFa = _FluxFn.apply(QW, WnB, QB, Blim, Bnf, g)
        gF = [gFa[5 * D:5 * D + 5] for D in range(3)]
        mF = [mFa[3 * D:3 * D + 3] for D in range(3)]
    for D in ([] if g.cuda_flux else range(3)):
        r = fr[D]
        T = [win(g.Tf[n + 9 * D], r) for n in range(9)]
        fa = win(A[D], r)
        Vi = central8([win(g.vol, r, unit(D, n - 4)) for n in range(8)])
        Bn = win(Bnf[D], r)
        Mag = [lrs_from_qdv(P, [win(QB[x], r, unit(D, n - 4)) for n in range(8)],
                            [win(Blim[x], r, unit(D, m - 2)) for m in range(4)], Vi) for x in range(3)]
        Wlr = [lrs_from_qdv(P, [win(QW[v], r, unit(D, n - 4)) for n in range(8)],
                            [win(WnB[v], r, unit(D, m - 2)) for m in range(4)], Vi) for v in range(5)]
        mFx = [torch.zeros_like(fa) for _ in range(3)]
        gFv = [torch.zeros_like(fa) for _ in range(5)]
        dW = [torch.zeros_like(fa) for _ in range(5)]
        VaD = torch.zeros_like(fa)
        if g.bg is not None:
            B0f = [win(g.bg["fcB0"][x + 3 * D], r).to(fa.dtype) for x in range(3)]
            B0n = (win(g.bg["bFlux0"][D], r) / win(A[D], r).double()).to(fa.dtype)
        for side, sgn in ((0, -1.0), (1, 1.0)):
            Wq = [Wlr[v][side] for v in range(5)]
            Bq = [Mag[x][side] for x in range(3)]
            # MagKinFlux (stress.F90:513-599), Boris off
            Dq, Pr = Wq[0], Wq[4]
            dPb = 0.5 * (Bq[0] * Bq[0] + Bq[1] * Bq[1] + Bq[2] * Bq[2])
            if g.bg is not None:
                sx, sy, sz = Bq[0] + B0f[0], Bq[1] + B0f[1], Bq[2] + B0f[2]
                Va2 = (sx * sx + sy * sy + sz * sz) / Dq
            else:
                Va2 = 2.0 * dPb / Dq
            Vn = T[0] * Wq[1] + T[1] * Wq[2] + T[2] * Wq[3]
            lam = 1.0 / (2.0 * Pr / Dq + Va2)
            Vn0 = 0.5 * torch.special.erfc(sgn * torch.sqrt(lam) * Vn)
            VaD = VaD + 0.5 * safe_sqrt(Va2)
            for x in range(3):
                mFx[x] = mFx[x] + Vn0 * (dPb * T[x] - Bq[x] * Bn)
            if g.bg is not None:
                BdB0 = B0f[0] * Bq[0] + B0f[1] * Bq[1] + B0f[2] * Bq[2]
                for x in range(3):
                    mFx[x] = mFx[x] + Vn0 * (-(B0f[x] * Bn) - Bq[x] * B0n + BdB0 * T[x])
            # GasKinFlux (stress.F90:432-511)
            Vx, Vy, Vz = Wq[1], Wq[2], Wq[3]
            Eg = 0.5 * Dq * (Vx * Vx + Vy * Vy + Vz * Vz) + Pr / gm1
            lam = Dq / (2.0 * Pr)
            Vn = T[0] * Vx + T[1] * Vy + T[2] * Vz
            Vt1 = T[3] * Vx + T[4] * Vy + T[5] * Vz
            Vt2 = T[6] * Vx + T[7] * Vy + T[8] * Vz
            Vn0 = 0.5 * torch.special.erfc(sgn * torch.sqrt(lam) * Vn)
            Vn1 = Vn * Vn0 - 0.5 * sgn * torch.exp(-(lam * Vn * Vn)) / torch.sqrt(PI * lam)
            gFv[0] = gFv[0] + Dq * Vn1
            gFv[4] = gFv[4] + (Eg + 0.5 * Pr) * Vn1 + 0.5 * Pr * Vn0 * Vn
            fMn = Dq * Vn * Vn1 + Pr * Vn0
            fMt1 = Dq * Vt1 * Vn1
            fMt2 = Dq * Vt2 * Vn1
            gFv[1] = gFv[1] + (T[0] * fMn + T[3] * fMt1 + T[6] * fMt2)
            gFv[2] = gFv[2] + (T[1] * fMn + T[4] * fMt1 + T[7] * fMt2)
            gFv[3] = gFv[3] + (T[2] * fMn + T[5] * fMt1 + T[8] * fMt2)
            dW[0] = dW[0] + sgn * Dq
            dW[1] = dW[1] + sgn * Dq * Vx
            dW[2] = dW[2] + sgn * Dq * Vy
            dW[3] = dW[3] + sgn * Dq * Vz
            dW[4] = dW[4] + sgn * Eg
        mF.append(put(torch.zeros_like(cur["B"]), r, torch.stack([fa * mFx[x] for x in range(3)])))
        gF.append(put(zeros5, r, torch.stack([fa * (gFv[v] - 1.0 * P.cHogH * VaD * dW[v]) for v in range(5)])))

    # --- applyUpdate: E2Flux on the active faces, then the cells
    if g.cuda_flux:
        Gas, mfn = _UpdateFn.apply(cur["Gas"], cur["mf"], Ea, gFa, mFa, g, dt)
    else:
        Gas, mfn = _update_torch(g, cur, E, gF, mF, dt)

    # --- EnforceBCs: inner sphere and solar wind in place, then the gathers
    # (periodic, zero-gradient J), then the final bFlux2Fld
    if P.bc[0] in (3, 6) or P.bc[1] in (2, 4):
        if g.cuda_flux:
            Gas, mfn = _ISideFn.apply(Gas, mfn, g.bxyz(mfn), g.inflow, g)
        else:
            Gas, mfn = _iside_bcs(g, Gas, mfn, g.bxyz(mfn))
    shp = Gas.shape
    Gas = _GatherFn.apply(Gas.reshape(5, -1), g.bc_src[-1], g.bc_adj[-1]).reshape(shp)
    mfs = mfn.reshape(3, -1)
    mfn = torch.stack([_GatherFn.apply(mfs[d:d + 1], g.bc_src[d], g.bc_adj[d])[0] for d in range(3)]).reshape(mfn.shape)
    return {"Gas": Gas, "mf": mfn, "B": g.bxyz(mfn)}


def _flux_params(g: Grid):
    from mage_b200.gamera import GamParams
    P = g.P
    gp = GamParams(P.Nip, P.Njp, P.Nkp, gamma=P.gamma, CFL=P.CFL, pdmb=P.pdmb, Vd0=P.Vd0, cHogH=P.cHogH,
                   dFloor=P.dFloor, pFloor=P.pFloor, doBackground=g.bg is not None)
    return gp.to_c()


class _FluxFn(torch.autograd.Function):
    """CalcStress on the GPU (gam_flux_forward) with the hand-written adjoint
    (gam_flux_adjoint) as its backward."""

    @staticmethod
    def forward(ctx, QW, Wn, QB, Blim, Bnf, g):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        ins = [t.contiguous() for t in (QW, Wn, QB, Blim, Bnf)]
        shp = g.face.shape[1:]
        gF = torch.zeros((15,) + tuple(shp), dtype=QW.dtype, device=QW.device)
        mF = torch.zeros((9,) + tuple(shp), dtype=QW.dtype, device=QW.device)
        p = _flux_params(g)
        bg = g.bg
        geo = [g.vol.contiguous(), g.face.contiguous(), g.Tf.contiguous()]
        fc = bg["fcB0"].contiguous().data_ptr() if bg is not None else None
        bf = bg["bFlux0"].contiguous().data_ptr() if bg is not None else None
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = L.gam_flux_forward(C.byref(p), int(QW.dtype == torch.float32), *[C.c_void_p(t.data_ptr()) for t in ins],
                                *[C.c_void_p(t.data_ptr()) for t in geo],
                                C.cast(C.c_void_p(fc), C.POINTER(C.c_double)) if fc else None,
                                C.cast(C.c_void_p(bf), C.POINTER(C.c_double)) if bf else None,
                                C.c_void_p(gF.data_ptr()), C.c_void_p(mF.data_ptr()), st)
        if rc != 0:
            raise RuntimeError(f"gam_flux_forward failed ({rc})")
        ctx.save_for_backward(*ins)
        ctx.g = g
        return gF, mF

    @staticmethod
    def backward(ctx, dgF, dmF):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        g = ctx.g
        ins = ctx.saved_tensors
        dgF = torch.zeros_like(ins[0][:1]).expand(15, *ins[0].shape[1:]).contiguous() if dgF is None else dgF.contiguous()
        dmF = torch.zeros_like(ins[0][:1]).expand(9, *ins[0].shape[1:]).contiguous() if dmF is None else dmF.contiguous()
        outs = [torch.zeros_like(t) for t in ins]
        p = _flux_params(g)
        bg = g.bg
        geo = [g.vol.contiguous(), g.face.contiguous(), g.Tf.contiguous()]
        fc = bg["fcB0"].contiguous().data_ptr() if bg is not None else None
        bf = bg["bFlux0"].contiguous().data_ptr() if bg is not None else None
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = L.gam_flux_adjoint(C.byref(p), int(ins[0].dtype == torch.float32),
                                *[C.c_void_p(t.data_ptr()) for t in ins], *[C.c_void_p(t.data_ptr()) for t in geo],
                                C.cast(C.c_void_p(fc), C.POINTER(C.c_double)) if fc else None,
                                C.cast(C.c_void_p(bf), C.POINTER(C.c_double)) if bf else None,
                                C.c_void_p(dgF.data_ptr()), C.c_void_p(dmF.data_ptr()),
                                *[C.c_void_p(t.data_ptr()) for t in outs], st)
        if rc != 0:
            raise RuntimeError(f"gam_flux_adjoint failed ({rc})")
        return (*outs, None)


def _ptr(t):
    import ctypes as C
    return C.c_void_p(t.data_ptr())


class _EFieldFn(torch.autograd.Function):
    """CalcElecField on the GPU (gam_efield_forward: Mom2Face + the edge EMF
    kernels) with the hand-written adjoint (gam_efield_adjoint) as backward."""

    @staticmethod
    def forward(ctx, Dh, abh, bn, VdV, g, dt):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        ins = [t.contiguous() for t in (Dh, abh, bn, VdV)]
        shp = tuple(g.face.shape[1:])
        AVf = torch.zeros((9,) + shp, dtype=abh.dtype, device=abh.device)
        E = torch.zeros((3,) + shp, dtype=abh.dtype, device=abh.device)
        p = _flux_params(g)
        geo = [g.vol.contiguous(), g.face.contiguous(), g.edge.contiguous(), g.Te.contiguous(), g.Teb.contiguous()]
        eb = g.bg["edgB0"].contiguous().data_ptr() if g.bg is not None else None
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = L.gam_efield_forward(C.byref(p), int(abh.dtype == torch.float32), *[_ptr(t) for t in ins],
                                  *[_ptr(t) for t in geo], C.cast(C.c_void_p(eb), C.POINTER(C.c_double)) if eb else None,
                                  float(dt), _ptr(AVf), _ptr(E), st)
        if rc != 0:
            raise RuntimeError(f"gam_efield_forward failed ({rc})")
        ctx.save_for_backward(*ins)
        ctx.g, ctx.dt = g, dt
        return E

    @staticmethod
    def backward(ctx, dE):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        g = ctx.g
        ins = ctx.saved_tensors
        shp = tuple(g.face.shape[1:])
        dE = dE.contiguous()
        outs = [torch.zeros_like(t) for t in ins]
        AVf = torch.zeros((9,) + shp, dtype=ins[1].dtype, device=ins[1].device)
        dAVf = torch.zeros((3,) + shp, dtype=ins[1].dtype, device=ins[1].device)
        p = _flux_params(g)
        geo = [g.vol.contiguous(), g.face.contiguous(), g.edge.contiguous(), g.Te.contiguous(), g.Teb.contiguous()]
        eb = g.bg["edgB0"].contiguous().data_ptr() if g.bg is not None else None
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = L.gam_efield_adjoint(C.byref(p), int(ins[1].dtype == torch.float32), *[_ptr(t) for t in ins],
                                  *[_ptr(t) for t in geo], C.cast(C.c_void_p(eb), C.POINTER(C.c_double)) if eb else None,
                                  float(ctx.dt), _ptr(AVf), _ptr(dE), *[_ptr(t) for t in outs], _ptr(dAVf), st)
        if rc != 0:
            raise RuntimeError(f"gam_efield_adjoint failed ({rc})")
        return (*outs, None, None)


def _vp(ptrs):
    import ctypes as C
    arr = (C.c_void_p * len(ptrs))(*[C.c_void_p(x) if x else None for x in ptrs])
    return arr


class _PredictFn(torch.autograd.Function):
    """Predictor on the GPU (gam_predict_stage: the product step's predictor
    kernel) with its hand-written adjoint as backward."""

    @staticmethod
    def forward(ctx, cG, cF, oG, oF, g, pdt, odt):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        st = [t.contiguous() for t in (cG, cF, oG, oF)]
        z5, z3, z1 = (torch.zeros_like(cG), torch.zeros_like(cF), torch.zeros_like(g.vol))
        outs = [z5, z5.clone(), z1, torch.zeros_like(cF), torch.zeros_like(cF), torch.zeros_like(cF),
                torch.zeros_like(cF), torch.zeros_like(cF)]
        geo = _geo_ptrs(g)
        rc = L.gam_predict_stage(C.byref(_flux_params(g)), int(cG.dtype == torch.float32),
                                 _vp([t.data_ptr() for t in st]), _vp(geo), float(pdt), float(odt),
                                 _vp([t.data_ptr() for t in outs]), None, None, None,
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gam_predict_stage failed ({rc})")
        ctx.save_for_backward(*st)
        ctx.g, ctx.pdt, ctx.odt = g, pdt, odt
        return tuple(outs)

    @staticmethod
    def backward(ctx, *douts):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        g = ctx.g
        st = ctx.saved_tensors
        shapes = [st[0], st[0], g.vol, st[1], st[1], st[1], st[1], st[1]]
        din = [torch.zeros_like(ref) if d is None else d.contiguous() for d, ref in zip(douts, shapes)]
        dst = [torch.zeros_like(t) for t in st]
        aB = torch.zeros_like(st[1])
        rc = L.gam_predict_stage(C.byref(_flux_params(g)), int(st[0].dtype == torch.float32),
                                 _vp([t.data_ptr() for t in st]), _vp(_geo_ptrs(g)), float(ctx.pdt), float(ctx.odt),
                                 None, _vp([t.data_ptr() for t in din]), C.c_void_p(aB.data_ptr()),
                                 _vp([t.data_ptr() for t in dst]), C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gam_predict_stage (adjoint) failed ({rc})")
        return (*dst, None, None, None)


def _geo_ptrs(g: Grid):
    f32 = g.dtype == torch.float32
    return [g.vol.data_ptr(), g.face.data_ptr(), g.xfc.data_ptr(), g.xyzcc.data_ptr(), g.dxf.data_ptr() if f32 else 0]


class _UpdateFn(torch.autograd.Function):
    """applyUpdate on the GPU (gam_update_stage: the product step's face and
    cell update kernels) with its hand-written adjoint as backward."""

    @staticmethod
    def forward(ctx, cG, cF, E, gF, mF, g, dt):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        ins = [t.contiguous() for t in (cG, cF, E, gF, mF)]
        nG, nF, nB = torch.zeros_like(cG), torch.zeros_like(cF), torch.zeros_like(cF)
        f32 = g.dtype == torch.float32
        geo = [g.vol.data_ptr(), g.xfc.data_ptr(), g.xyzcc.data_ptr(), g.dxf.data_ptr() if f32 else 0]
        dp = g.bg["dpB0"].contiguous().data_ptr() if g.bg is not None else None
        rc = L.gam_update_stage(C.byref(_flux_params(g)), int(f32), _vp([t.data_ptr() for t in ins]), _vp(geo),
                                C.cast(C.c_void_p(dp), C.POINTER(C.c_double)) if dp else None, float(dt),
                                _vp([nG.data_ptr(), nF.data_ptr(), nB.data_ptr()]), None, None, None, None,
                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gam_update_stage failed ({rc})")
        ctx.save_for_backward(*ins)
        ctx.g, ctx.dt = g, dt
        return nG, nF

    @staticmethod
    def backward(ctx, dG, dF):
        import ctypes as C
        from mage_b200.gamera import load_library
        L = load_library()
        g = ctx.g
        ins = ctx.saved_tensors
        dG = torch.zeros_like(ins[0]) if dG is None else dG.contiguous()
        dF = torch.zeros_like(ins[1]) if dF is None else dF.contiguous()
        dst = [torch.zeros_like(t) for t in ins]
        sU, sM = torch.zeros_like(ins[0]), torch.zeros_like(ins[1])
        f32 = g.dtype == torch.float32
        geo = [g.vol.data_ptr(), g.xfc.data_ptr(), g.xyzcc.data_ptr(), g.dxf.data_ptr() if f32 else 0]
        dp = g.bg["dpB0"].contiguous().data_ptr() if g.bg is not None else None
        rc = L.gam_update_stage(C.byref(_flux_params(g)), int(f32), _vp([t.data_ptr() for t in ins]), _vp(geo),
                                C.cast(C.c_void_p(dp), C.POINTER(C.c_double)) if dp else None, float(ctx.dt), None,
                                _vp([dG.data_ptr(), dF.data_ptr()]), C.c_void_p(sU.data_ptr()),
                                C.c_void_p(sM.data_ptr()), _vp([t.data_ptr() for t in dst]),
                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gam_update_stage (adjoint) failed ({rc})")
        return (*dst, None, None)


def _iside_struct(g: Grid, inflow=None):
    """gam_iside for the grid's I boundaries, and the tensors it points to."""
    from mage_b200.gamera import ISide
    P = g.P
    s, keep = ISide(), []
    if P.bc[0] == 6:
        w = (g.inflow if inflow is None else inflow).detach().double().cpu().tolist()
        for q in range(8):
            s.inflow[q] = w[q]
    if P.bc[1] == 4:
        W = g.wind
        for q in range(8):
            s.wind[q] = float(W["state"][q])
        keep = [W["wC"].contiguous()] + [W[f"wF{d}"].contiguous() for d in range(3)] + \
               [W[f"sF{d}"].contiguous() for d in range(3)]
        s.wC = keep[0].data_ptr()
        for d in range(3):
            s.wF[d] = keep[1 + d].data_ptr()
            s.sF[d] = keep[4 + d].data_ptr()
    return s, keep


def _bc_params(g: Grid):
    from mage_b200.gamera import GamParams
    P = g.P
    return GamParams(P.Nip, P.Njp, P.Nkp, gamma=P.gamma, CFL=P.CFL, pdmb=P.pdmb, Vd0=P.Vd0, cHogH=P.cHogH,
                     dFloor=P.dFloor, pFloor=P.pFloor, doBackground=g.bg is not None, bc=tuple(P.bc)).to_c()


class _ISideFn(torch.autograd.Function):
    """The non-periodic I boundaries (the inflow or SphIn inside, zeroGrad_obcI
    or the constant wind outside) by gam_iside_fill, with gam_iside_adjoint as
    backward; _iside_bcs is the same fill as PyTorch expressions. B is the
    field of the update's fluxes, inflow the inflow state (or None)."""

    @staticmethod
    def forward(ctx, Gas, mf, B, inflow, g):
        import ctypes as C
        from mage_b200.gamera import GamError, load_library
        L = load_library()
        Gas, mf, B = Gas.contiguous().clone(), mf.contiguous().clone(), B.contiguous()
        s, keep = _iside_struct(g, inflow)
        f32 = int(g.dtype == torch.float32)
        geo = _vp([g.face.data_ptr(), g.Tf.data_ptr()])
        rc = L.gam_iside_fill(C.byref(_bc_params(g)), f32, geo, C.byref(s), C.c_void_p(B.data_ptr()),
                              C.c_void_p(Gas.data_ptr()), C.c_void_p(mf.data_ptr()),
                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise GamError(rc, "gam_iside_fill failed")
        ctx.save_for_backward(Gas, B)
        ctx.g, ctx.inflow = g, inflow
        return Gas, mf

    @staticmethod
    def backward(ctx, dG, dM):
        import ctypes as C
        from mage_b200.gamera import GamError, load_library
        L = load_library()
        g = ctx.g
        Gas, B = ctx.saved_tensors
        dG = torch.zeros_like(Gas) if dG is None else dG.contiguous().clone()
        dM = torch.zeros_like(B) if dM is None else dM.contiguous().clone()
        dB = torch.zeros_like(B)
        dw = None
        if ctx.inflow is not None and ctx.needs_input_grad[3]:
            dw = torch.zeros(8, dtype=g.dtype, device=Gas.device)
        s, keep = _iside_struct(g, ctx.inflow)
        f32 = int(g.dtype == torch.float32)
        geo = _vp([g.face.data_ptr(), g.Tf.data_ptr()])
        rc = L.gam_iside_adjoint(C.byref(_bc_params(g)), f32, geo, C.byref(s), C.c_void_p(Gas.data_ptr()),
                                 C.c_void_p(B.data_ptr()), C.c_void_p(dG.data_ptr()), C.c_void_p(dM.data_ptr()),
                                 C.c_void_p(dB.data_ptr()), C.c_void_p(dw.data_ptr()) if dw is not None else None,
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise GamError(rc, "gam_iside_adjoint failed")
        return dG, dM, dB, dw, None


class WholeStep:
    """One stepGamera and its adjoint as one C call each (gam_step_fwd_save,
    gam_step_adj, or their _iside variants): the stage kernels of the classes
    above plus the step's boundaries and bFlux2Fld on the device, without
    autograd. Periodic K, periodic or zero-gradient J, periodic I or the
    inflow / SphIn inside with zeroGrad_obcI / the wind outside; the work
    area (gam_step_work_bytes) holds one step's intermediate arrays."""

    def __init__(self, g: Grid):
        import ctypes as C
        from mage_b200.gamera import GamError, GamParams, load_library
        P = g.P
        self.g, self.L = g, load_library()
        self.p = GamParams(P.Nip, P.Njp, P.Nkp, gamma=P.gamma, CFL=P.CFL, pdmb=P.pdmb, Vd0=P.Vd0, cHogH=P.cHogH,
                           dFloor=P.dFloor, pFloor=P.pFloor, doBackground=g.bg is not None, bc=tuple(P.bc)).to_c()
        self.f32 = int(g.dtype == torch.float32)
        nb = C.c_int64()
        rc = self.L.gam_step_work_bytes(C.byref(self.p), self.f32, C.byref(nb))
        if rc != 0:
            raise GamError(rc, "gam_step_work_bytes: the whole-step adjoint does not cover these parameters")
        self.work = torch.empty(nb.value, dtype=torch.uint8, device=g.device)
        self._geo = [g.vol, g.face, g.xfc, g.xyzcc, g.dxf if self.f32 else None, g.edge, g.Te, g.Teb, g.Tf]
        self._geo = [t.contiguous() if t is not None else None for t in self._geo]
        self.geo = _vp([t.data_ptr() if t is not None else 0 for t in self._geo])
        self.bg = None
        if g.bg is not None:
            self._bg = [g.bg[k].contiguous() for k in ("fcB0", "bFlux0", "edgB0", "dpB0")]
            self.bg = _vp([t.data_ptr() for t in self._bg])

    def _st(self, cur, old):
        ts = [t.contiguous() for t in (cur["Gas"], cur["mf"], old["Gas"], old["mf"])]
        return ts, _vp([t.data_ptr() for t in ts])

    def forward(self, cur: dict, old: dict, dt: float, odt: float) -> dict:
        """State after the step (gam_step_fwd_save); cur/old as for step()."""
        import ctypes as C
        from mage_b200.gamera import GamError
        ts, st = self._st(cur, old)
        nxt = {"Gas": torch.empty_like(ts[0]), "mf": torch.empty_like(ts[1]), "B": torch.empty_like(ts[1])}
        out = _vp([nxt[k].data_ptr() for k in ("Gas", "mf", "B")])
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        if self.g.P.bc[0] != 0:
            s, keep = _iside_struct(self.g)
            rc = self.L.gam_step_fwd_save_iside(C.byref(self.p), self.f32, self.geo, self.bg, C.byref(s), st,
                                                float(dt), float(odt), out, C.c_void_p(self.work.data_ptr()), stream)
        else:
            rc = self.L.gam_step_fwd_save(C.byref(self.p), self.f32, self.geo, self.bg, st, float(dt), float(odt),
                                          out, C.c_void_p(self.work.data_ptr()), stream)
        if rc != 0:
            raise GamError(rc, "gam_step_fwd_save failed")
        return nxt

    def adjoint(self, cur: dict, old: dict, dt: float, odt: float, dnxt: dict, acc=None, saved: bool = False,
                dinflow=None):
        """Adjoints (dcurGas, dcurMf, doldGas, doldMf) of the step's start for
        the adjoints dnxt = {"Gas", "mf", "B" (optional)} of its result, added
        to acc (four tensors) when given (gam_step_adj); with the inflow
        boundary, the inflow state's adjoints are added into dinflow (8
        values on the device) when given."""
        import ctypes as C
        from mage_b200.gamera import GamError
        ts, st = self._st(cur, old)
        dn = [dnxt["Gas"].contiguous(), dnxt["mf"].contiguous()]
        dB = dnxt.get("B")
        dB = dB.contiguous() if dB is not None else None
        dst = [a.contiguous() for a in acc] if acc is not None else [torch.zeros_like(t) for t in ts]
        dnp = _vp([dn[0].data_ptr(), dn[1].data_ptr(), dB.data_ptr() if dB is not None else 0])
        dsp = _vp([t.data_ptr() for t in dst])
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        if self.g.P.bc[0] != 0:
            s, keep = _iside_struct(self.g)
            rc = self.L.gam_step_adj_iside(C.byref(self.p), self.f32, self.geo, self.bg, C.byref(s), st, float(dt),
                                           float(odt), int(saved), dnp, dsp,
                                           C.c_void_p(dinflow.data_ptr()) if dinflow is not None else None,
                                           C.c_void_p(self.work.data_ptr()), stream)
        else:
            rc = self.L.gam_step_adj(C.byref(self.p), self.f32, self.geo, self.bg, st, float(dt), float(odt),
                                     int(saved), dnp, dsp, C.c_void_p(self.work.data_ptr()), stream)
        if rc != 0:
            raise GamError(rc, "gam_step_adj failed")
        return dst


def _face_proj(g: Grid, d: int, idx, B):
    """face * (n . B) on face d at box index idx (zeroGrad_obcI, bcs.F90:842-844)."""
    t = [g.Tf[q + 9 * d][idx] for q in range(3)]
    return g.face[d][idx] * (B[0] * t[0] + B[1] * t[1] + B[2] * t[2])


def _iside_bcs(g: Grid, Gas, mf, B):
    """SphIn (bcs.F90:934-957) or the uniform inflow on the inner I side, the
    constant-wind WindBC (apps/wind.F90:206-374) or zeroGrad_obcI
    (bcs.F90:820-850) on the outer one, on their 4 ghost layers; B is the Bxyz
    of the updated state."""
    P = g.P
    Ni, Nj, Nk = g.Ni, g.Nj, g.Nk
    ip = G + P.Nip - 1
    cellsJK = (slice(0, Nk), slice(0, Nj))
    if P.bc[0] == 6:
        w = g.inflow
        gC = cell_p2c(P, [w[0], w[2], w[3], w[4], w[1]])
        Gas = Gas.clone()
        mf = mf.clone()
        for n in range(1, 5):
            for v in range(5):
                Gas[v, :Nk, :Nj, G - n] = gC[v]
            for d in range(3):
                mf[d, :Nk, :Nj, G - n] = _face_proj(g, d, cellsJK + (G - n,), (w[5], w[6], w[7]))
    if P.bc[1] == 2:
        Bc = [B[x][cellsJK + (ip,)] for x in range(3)]
        gsrc = Gas[:, :Nk, :Nj, ip].clone()
        Gas = Gas.clone()
        mf = mf.clone()
        for n in range(1, 5):
            Gas[:, :Nk, :Nj, ip + n] = gsrc
            mf[0, :Nk, :Nj, ip + n + 1] = _face_proj(g, 0, cellsJK + (ip + n + 1,), Bc)
            for d in (1, 2):
                mf[d, :Nk, :Nj, ip + n] = _face_proj(g, d, cellsJK + (ip + n,), Bc)
    if P.bc[0] == 3:
        gsrc = Gas[:, :Nk, :Nj, G].clone()
        fsrc = mf[:, :Nk, :Nj, G].clone()
        Gas = Gas.clone()
        mf = mf.clone()
        for n in range(1, 5):
            Gas[:, :Nk, :Nj, G - n] = gsrc
            mf[:, :Nk, :Nj, G - n] = fsrc
    if P.bc[1] == 4:
        W = g.wind
        w = W["state"]
        gC = [Gas[v][cellsJK + (ip,)] for v in range(5)]
        Bin = [B[x][cellsJK + (ip,)] for x in range(3)]
        gW_in = cell_c2p(P, gC)
        # Con2Fast (gamutils.F90:238-269)
        rho = rmax(gC[0], torch.full_like(gC[0], P.dFloor))
        Vx, Vy, Vz = gC[1] / rho, gC[2] / rho, gC[3] / rho
        KinE = 0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz)
        Pr = rmax((P.gamma - 1) * (gC[4] - KinE), torch.full_like(rho, P.pFloor))
        Cs = torch.sqrt(P.gamma * Pr / rho)
        MagB = safe_sqrt(Bin[0] * Bin[0] + Bin[1] * Bin[1] + Bin[2] * Bin[2])
        Va = MagB / torch.sqrt(gC[0])
        Cx = torch.sqrt(Cs * Cs + Va * Va)
        nH = [g.Tf[q][cellsJK + (ip + 1,)] for q in range(3)]
        V = [gW_in[1], gW_in[2], gW_in[3]]
        dn = V[0] * nH[0] + V[1] * nH[1] + V[2] * nH[2]
        fix = _see(dn < Cx)  # MinMach = 1
        V = [torch.where(fix, V[x] - dn * nH[x] + Cx * nH[x], V[x]) for x in range(3)]
        fin = [mf[0, :, :, ip + 1].clone(), mf[1, :, :, ip].clone(), mf[2, :, :, ip].clone()]
        Gas = Gas.clone()
        mf = mf.clone()
        for n in range(1, 5):
            wSW = W["wC"][:, :, n - 1]
            wMHD = 1.0 - wSW
            sw = (wSW > TINY).to(wSW.dtype)
            mh = (wMHD > TINY).to(wSW.dtype)
            gW_sw = [sw * w[0], sw * w[2], sw * w[3], sw * w[4], sw * w[1]]
            gWi = [mh * gW_in[0], mh * V[0], mh * V[1], mh * V[2], mh * gW_in[4]]
            gW = [wSW * gW_sw[v] + wMHD * gWi[v] for v in range(5)]
            gCn = cell_p2c(P, gW)
            for v in range(5):
                Gas[v, :Nk, :Nj, ip + n] = gCn[v]
            wI = W["wF0"][:, :, n - 1]
            mf[0, :, :, ip + n + 1] = wI * W["sF0"][:, :, n - 1] + (1.0 - wI) * fin[0]
            for d in (1, 2):
                wd = W[f"wF{d}"][:, :, n - 1]
                mf[d, :, :, ip + n] = wd * W[f"sF{d}"][:, :, n - 1] + (1.0 - wd) * fin[d]
    return Gas, mf


def run(g: Grid, cur: dict, old: dict, dt: float, nsteps: int, odt0: float | None = None):
    """nsteps fixed-dt steps; the AB2 spacing is odt0 for the first step
    (time - otime of the start), dt afterwards. Returns (State, oState)."""
    odt = dt if odt0 is None else odt0
    for _ in range(nsteps):
        nxt = step(g, cur, old, dt, odt)
        old, cur = cur, nxt
        odt = dt
    return cur, old


def loss_b2(g: Grid, state: dict, lo=0.6, hi=0.8):
    """Sum of |B|^2 over the active cells whose centre lies in [lo, hi]^3."""
    P = g.P
    act = (G, G + P.Nip - 1, G, G + P.Njp - 1, G, G + P.Nkp - 1)
    xc = win(g.xyzcc, act)
    m = ((xc >= lo) & (xc <= hi)).all(dim=0)
    B = win(state["B"], act)
    return ((B * B).sum(dim=0) * m).sum()


def loss_and_grad(g: Grid, Gas0, mf0, dt: float, nsteps: int, seg: int | None = None, lossf=loss_b2,
                  per_step: bool = False, params=None):
    """Loss after nsteps from the start State = oState = (Gas0, mf0, bxyz(mf0))
    (otime = time - dt) and its gradient w.r.t. Gas0 and mf0; with params (a
    list of tensors the grid's boundaries use every step, e.g. [g.inflow])
    also the gradients w.r.t. those, as a fourth result.

    Checkpointing: the forward sweep keeps only the (State, oState) pair at the
    start of each segment of seg steps (default ~sqrt(nsteps)); the reverse
    sweep recomputes one segment at a time and carries the adjoint of the pair
    backwards. per_step: within a segment, recompute and store the states
    without a graph, then differentiate one step at a time (two-level
    checkpointing: memory of one step's graph plus seg states)."""
    seg = seg or max(1, int(round(nsteps ** 0.5)))
    with torch.no_grad():
        cur = {"Gas": Gas0, "mf": mf0, "B": g.bxyz(mf0)}
        old = dict(cur)
        ckpt = []
        n = 0
        while n < nsteps:
            ckpt.append((n, {k: v.clone() for k, v in cur.items()}, {k: v.clone() for k, v in old.items()}))
            m = min(seg, nsteps - n)
            cur, old = run(g, cur, old, dt, m)
            n += m
        del cur, old
    params = list(params or [])
    pleaves = [p.detach().requires_grad_(True) for p in params]
    swaps = [(k, getattr(g, k)) for k in ("inflow",) if any(getattr(g, k) is p for p in params)]
    for k, p in swaps:
        setattr(g, k, pleaves[[id(q) for q in params].index(id(p))])
    pacc = [torch.zeros_like(p) for p in pleaves]
    lam_cur = lam_old = None
    loss_val = None
    for idx in range(len(ckpt) - 1, -1, -1):
        n0, c0, o0 = ckpt.pop()
        m = min(seg, nsteps - n0)
        if per_step:
            sts = [(c0, o0)]
            with torch.no_grad():
                c, o = c0, o0
                for _ in range(m - 1):
                    c, o = run(g, c, o, dt, 1)
                    sts.append((c, o))
            units = [(n0 + k, sts[k][0], sts[k][1], 1) for k in range(m - 1, -1, -1)]
        else:
            units = [(n0, c0, o0, m)]
        for ns, cs, os_, mm in units:
            first = ns == 0
            if first:
                G0 = Gas0.detach().clone().requires_grad_(True)
                F0 = mf0.detach().clone().requires_grad_(True)
                c = {"Gas": G0, "mf": F0, "B": g.bxyz(F0)}
                o = c
                leaves = [G0, F0]
            else:
                c = {k: v.detach().clone().requires_grad_(True) for k, v in cs.items()}
                o = {k: v.detach().clone().requires_grad_(True) for k, v in os_.items()}
                leaves = [c[k] for k in ("Gas", "mf", "B")] + [o[k] for k in ("Gas", "mf", "B")]
            leaves = leaves + pleaves
            with torch.enable_grad():
                ce, oe = run(g, c, o, dt, mm)
                if lam_cur is None:
                    L = lossf(g, ce)
                    loss_val = float(L.detach())
                    outs, grads = [L], [torch.ones_like(L)]
                else:
                    outs, grads = [], []
                    for k in ("Gas", "mf", "B"):
                        outs += [ce[k], oe[k]]
                        grads += [lam_cur[k], lam_old[k]]
                gl = torch.autograd.grad(outs, leaves, grads, allow_unused=True)
            gl = [torch.zeros_like(x) if gv is None else gv for x, gv in zip(leaves, gl)]
            if pleaves:
                pacc = [a + b for a, b in zip(pacc, gl[len(gl) - len(pleaves):])]
                gl = gl[:len(gl) - len(pleaves)]
            del ce, oe, outs, grads, c, o
            if first:
                for k, p in swaps:
                    setattr(g, k, p)
                if params:
                    return loss_val, gl[0], gl[1], pacc
                return loss_val, gl[0], gl[1]
            lam_cur = dict(zip(("Gas", "mf", "B"), gl[:3]))
            lam_old = dict(zip(("Gas", "mf", "B"), gl[3:]))
    raise AssertionError("unreachable")


def loss_and_grad_c(g: Grid, Gas0, mf0, dt: float, nsteps: int, seg: int | None = None, lossf=loss_b2,
                    params=None):
    """loss_and_grad through the whole-step C entry points: the same
    checkpointing (the (State, oState) pair at the start of each segment of
    seg steps), the segment's states recomputed with gam_step_fwd_save, then
    gam_step_adj one step at a time backwards; autograd only for the loss's
    own gradient. The adjoint of oState at step n is the adjoint of State at
    step n-1, so it seeds that step's accumulators. params = [g.inflow]
    also returns the loss's gradient w.r.t. the inflow state (the sum of
    every step's inflow adjoints), as a fourth result."""
    params = list(params or [])
    for q in params:
        assert q is g.inflow, "loss_and_grad_c differentiates w.r.t. the inflow state only"
    dw = torch.zeros(8, dtype=g.dtype, device=Gas0.device) if params else None
    ws = WholeStep(g)
    seg = seg or max(1, int(round(nsteps ** 0.5)))
    with torch.no_grad():
        cur = {"Gas": Gas0.contiguous(), "mf": mf0.contiguous(), "B": g.bxyz(mf0)}
        old = cur
        ckpt = []
        n = 0
        while n < nsteps:
            ckpt.append((n, cur, old))
            for _ in range(min(seg, nsteps - n)):
                cur, old = ws.forward(cur, old, dt, dt), cur
            n += min(seg, nsteps - n)
        fin = {k: v.detach().clone().requires_grad_(True) for k, v in cur.items()}
    with torch.enable_grad():
        L = lossf(g, fin)
        gl = torch.autograd.grad(L, [fin["Gas"], fin["mf"], fin["B"]], allow_unused=True)
    lam = {k: (torch.zeros_like(fin[k]) if v is None else v) for k, v in zip(("Gas", "mf", "B"), gl)}
    carry = None  # adjoint of the oState of the step after the current one
    with torch.no_grad():
        for n0, c0, o0 in reversed(ckpt):
            m = min(seg, nsteps - n0)
            sts = [(c0, o0)]
            for _ in range(m - 1):
                c, o = sts[-1]
                sts.append((ws.forward(c, o, dt, dt), c))
            for c, o in reversed(sts):
                acc = [torch.zeros_like(c["Gas"]), torch.zeros_like(c["mf"]), torch.zeros_like(o["Gas"]),
                       torch.zeros_like(o["mf"])]
                if carry is not None:
                    acc[0].add_(carry[0])
                    acc[1].add_(carry[1])
                d = ws.adjoint(c, o, dt, dt, lam, acc, dinflow=dw)
                lam = {"Gas": d[0], "mf": d[1]}
                carry = (d[2], d[3])
    # step 0 starts from State = oState = (Gas0, mf0)
    if params:
        return float(L.detach()), lam["Gas"] + carry[0], lam["mf"] + carry[1], [dw]
    return float(L.detach()), lam["Gas"] + carry[0], lam["mf"] + carry[1]
