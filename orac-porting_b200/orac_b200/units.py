"""ORAC internal units: amu, Angstrom, fs.

Restates setuns (src/setuns.f:34-48), the charge scaling of covchg
(src/covchg.f:37-39) and the Amber combination rule of covnb
(src/covnb.f, iz=0 branch).  Energies printed by ORAC are efact/1000 kJ/mol
per internal unit.
"""
import math

PI = 4.0 * math.atan(1.0)
AVOGAD = 6.022140857e23
BOLTZ = 1.38064852e-23
GASCON = 8.3144598
ELECHG = 1.60217662e-19
EPSO = 8.854187817e-12
UNITM = 1.0 / (AVOGAD * 1000.0)
UNITL = 1.0e-10
UNITT = 1.0e-15
UNITE = UNITM * (UNITL / UNITT) ** 2
UNITC = 4.0 * PI * EPSO * UNITL * UNITE / (ELECHG * ELECHG)
EFACT = UNITE * AVOGAD  # J/mol per internal energy unit
KJMOL = EFACT / 1000.0  # kJ/mol per internal energy unit

# covnb multiplies by a default-real literal 4.184 (single precision)
_F4184 = float.fromhex("0x1.0bc6a80000000p+2")  # float32(4.184) widened
assert abs(_F4184 - 4.184) < 1e-6


def charge_internal(q_e):
    """Electron charges -> ORAC internal charge units (covchg.f:37-39)."""
    return q_e / math.sqrt(UNITC)


def amber_pair(rmin_half_i, eps_i, rmin_half_j, eps_j):
    """(ecc12, ecc6) for one type pair, covnb.f amber branch.

    rmin_half is the prm file's Rmin/2 in Angstrom, eps in kcal/mol.
    """
    fact = 1.0 / (2.0 ** (1.0 / 6.0))
    qener = math.sqrt(abs(eps_i * eps_j))
    tmpi = 4.0 * 1000.0 * qener * _F4184 / (UNITE * AVOGAD)
    tmpj = ((rmin_half_i + rmin_half_j) * fact) ** 6
    return tmpi * tmpj * tmpj, tmpi * tmpj


def alchemy_rmin_epsm(rmin_half, eps_kcal):
    """Per-atom soft-core parameters, src/mtsmd.f:1298-1303:
    rmin = pnbd1 / 2**(1./6.) with the exponent a default-real (single
    precision) quotient, epsm = |pnbd2 * (1000 * 4.184 / efact)| with a
    single-precision 4.184, and rmin = 0.1 where epsm is zero."""
    import numpy as np

    sixth = float(np.float32(1.0) / np.float32(6.0))
    rmin = np.asarray(rmin_half, dtype=np.float64) / 2.0 ** sixth
    epsm = np.abs(np.asarray(eps_kcal, dtype=np.float64) * (1000.0 * _F4184 / EFACT))
    rmin = np.where(epsm == 0.0, 0.1, rmin)
    return rmin, epsm


def kinetic_temperature(ekin_internal, ndf):
    """Temperature in K from kinetic energy in internal units and degrees of freedom."""
    return 2.0 * ekin_internal * UNITE / (ndf * BOLTZ)
