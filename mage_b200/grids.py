"""Corner grids for the GAMERA step (host side, FP64).

Corner arrays use the reference's memory layout: Fortran
``xyz(isg:ieg+1, jsg:jeg+1, ksg:keg+1, 1:3)`` with i fastest, which in numpy
is a C-ordered array of shape ``(3, Nk+1, Nj+1, Ni+1)`` (component, k, j, i),
``Ni = Nip + 2*nG``, ``nG = 4``, and corner index ``i`` running from
``isg = 1 - nG`` to ``ieg + 1 = Nip + nG + 1``.
"""
from __future__ import annotations

import numpy as np

NG = 4


def _axis(n: int, lo: float, hi: float) -> np.ndarray:
    """Corner coordinates along one axis, init.F90:684-689 (genGridXML):
    ``x = min + (i-1)*dx`` with ``dx = (max-min)/N`` for i = isg .. ieg+1."""
    dx = (hi - lo) / n
    i = np.arange(1 - NG, n + NG + 2, dtype=np.float64)
    return lo + (i - 1.0) * dx


def uniform_corners(Nip: int, Njp: int, Nkp: int, bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0)) -> np.ndarray:
    """Uniform Cartesian corners (genGridXML without doCyl/doSph/doWarp)."""
    x1 = _axis(Nip, bounds[0], bounds[1])
    x2 = _axis(Njp, bounds[2], bounds[3])
    x3 = _axis(Nkp, bounds[4], bounds[5])
    xyz = np.empty((3, x3.size, x2.size, x1.size), dtype=np.float64)
    xyz[0] = x1[None, None, :]
    xyz[1] = x2[None, :, None]
    xyz[2] = x3[:, None, None]
    return xyz


def warped_periodic_corners(Nip: int, Njp: int, Nkp: int, amp: float = 0.05) -> np.ndarray:
    """Non-orthogonal curvilinear corners on the unit cube:
    ``x = xi + amp*s, y = eta + amp*s, z = zeta + amp*s`` with
    ``s = sin(2 pi xi) sin(2 pi eta) sin(2 pi zeta)``. The map commutes with unit
    shifts, so the grid is triply periodic; ghost corners use the same formula."""
    u = uniform_corners(Nip, Njp, Nkp)
    xi, eta, zeta = u[0], u[1], u[2]
    s = np.sin(2.0 * np.pi * xi) * np.sin(2.0 * np.pi * eta) * np.sin(2.0 * np.pi * zeta)
    return np.stack([xi + amp * s, eta + amp * s, zeta + amp * s]).astype(np.float64)


def dims(xyz: np.ndarray):
    """(Nip, Njp, Nkp) of a corner array."""
    _, nk1, nj1, ni1 = xyz.shape
    return ni1 - 1 - 2 * NG, nj1 - 1 - 2 * NG, nk1 - 1 - 2 * NG


def spherical_corners(Nr: int, Nth: int, Nph: int, r0: float = 2.0, r1: float = 30.0, th0: float = 0.05,
                      th1: float = float(np.pi) - 0.05) -> np.ndarray:
    """Spherical-polar corners: r log-spaced on [r0, r1], theta uniform on
    [th0, th1], phi uniform on [0, 2 pi) (periodic), x = r sin(th) cos(ph),
    y = r sin(th) sin(ph), z = r cos(th). Ghost corners continue the same
    formulas (as genGridXML does for doSph, init.F90:668-690)."""
    i = np.arange(1 - NG, Nr + NG + 2, dtype=np.float64)
    j = np.arange(1 - NG, Nth + NG + 2, dtype=np.float64)
    k = np.arange(1 - NG, Nph + NG + 2, dtype=np.float64)
    r = r0 * (r1 / r0) ** ((i - 1.0) / Nr)
    th = th0 + (th1 - th0) * (j - 1.0) / Nth
    ph = 2.0 * np.pi * (k - 1.0) / Nph
    R = r[None, None, :]
    TH = th[None, :, None]
    PH = ph[:, None, None]
    xyz = np.empty((3, k.size, j.size, i.size), dtype=np.float64)
    xyz[0] = R * np.sin(TH) * np.cos(PH)
    xyz[1] = R * np.sin(TH) * np.sin(PH)
    xyz[2] = R * np.cos(TH) * np.ones_like(PH)
    return xyz


def lfm_corners(Nr: int, Nth: int, Nph: int, r0: float = 2.0, r1: float = 30.0, th0: float = 0.0) -> np.ndarray:
    """LFM-style corners: spherical about the x axis, the polar angle th on
    [th0, pi - th0] from +x (j, the axis at js and je+1 when th0 = 0), the
    azimuth ph on [0, 2 pi) around x (k, periodic), r log-spaced on [r0, r1]
    (i): x = r cos(th), y = r sin(th) cos(ph), z = r sin(th) sin(ph). Ghost
    corners continue the formulas, so with th0 = 0 the ghosts across the axis
    fall on the cells that the pole boundary maps them to (mirrored j,
    k + Nph/2)."""
    i = np.arange(1 - NG, Nr + NG + 2, dtype=np.float64)
    j = np.arange(1 - NG, Nth + NG + 2, dtype=np.float64)
    k = np.arange(1 - NG, Nph + NG + 2, dtype=np.float64)
    r = r0 * (r1 / r0) ** ((i - 1.0) / Nr)
    th = th0 + (np.pi - 2.0 * th0) * (j - 1.0) / Nth
    ph = 2.0 * np.pi * (k - 1.0) / Nph
    R = r[None, None, :]
    TH = th[None, :, None]
    PH = ph[:, None, None]
    xyz = np.empty((3, k.size, j.size, i.size), dtype=np.float64)
    xyz[0] = R * np.cos(TH) * np.ones_like(PH)
    xyz[1] = R * np.sin(TH) * np.cos(PH)
    xyz[2] = R * np.sin(TH) * np.sin(PH)
    return xyz
