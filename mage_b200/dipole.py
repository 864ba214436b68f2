"""Dipole-in-wind set-up constants (the spherical magnetosphere workloads).

Code units follow the reference's Earth magnetosphere normalisation
(src/gamera/apps/msphutils.F90:19-36, src/base/planethelper.F90:96-123):
length 1 R_E, velocity 100 km/s, density 1 amu/cc, field 4.58 nT, pressure
1.67e-2 nPa, dipole moment M0 = -EarthM0g * 1e5 / 4.58 (EarthM0g =
0.2961737 G, src/base/kdefs.F90). The solar wind (rho = 5 /cc,
v = (-400, 0, 0) km/s, T = 1e5 K, IMF Bz = -5 nT) in those units:
"""
KB = 1.380649e-23          # J/K
P0_PA = 1.67e-2 * 1.0e-9   # code pressure unit [Pa]
V0_KMS = 100.0
B0_NT = 4.58
EARTH_M0G = 0.2961737

M0 = -EARTH_M0G * 1.0e5 / B0_NT


def wind_code_units(n_cc=5.0, vx_kms=-400.0, T_K=1.0e5, bz_nT=-5.0):
    """(rho, P, Vx, Vy, Vz, Bx, By, Bz) of a constant solar wind in code units."""
    P = n_cc * 1.0e6 * KB * T_K / P0_PA
    return (n_cc, P, vx_kms / V0_KMS, 0.0, 0.0, 0.0, 0.0, bz_nT / B0_NT)
