"""Checks of the oracle's bonded routines (fpbond, fpbend with Urey-Bradley,
fptors, fitors) on the CPU: forces are minus the gradient of the energy the
routine reports, energies have the closed forms of the reference routines,
and the torsion energy is the polynomial form of V cos(n phi).
"""
import math

import numpy as np
import pytest

import oracle
from orac_b200 import systems


def chain_system(nchain=24, seed=5):
    s = systems.polymer_in_water(nchain=nchain, nwat=8, box=24.0, nfft=(16, 16, 16), order=4, group_size=3,
                                 seed_chain=seed, name="chain24")
    rng = np.random.default_rng(seed)
    # impropers: half harmonic (potc > 0, phi0 = 1 rad), half cosine n = 2
    quads = np.array([(i + 1, i + 2, i + 3, i + 4) for i in range(0, nchain - 4, 3)], dtype=np.int32)
    k = len(quads)
    s.itors = quads
    s.itors_a = np.where(np.arange(k) % 2 == 0, 1.0, 2.0)
    s.itors_b = rng.uniform(0.5, 2.0, k) * 4184.0 / 6.022140857e23 / 1e-20 * 1e-3
    s.itors_c = np.where(np.arange(k) % 2 == 0, 1.0, 0.0)
    # Urey-Bradley on every bend
    s.bend_ub_r0 = np.full(len(s.bends), 2.5)
    s.bend_ub_k = np.full(len(s.bends), 0.3 * s.bend_k[0])
    # mixed torsion multiplicities and phases
    s.tors_n = np.array([[1.0, -2.0, 3.0, -3.0, 4.0, 6.0][i % 6] for i in range(len(s.tors))])
    # move the chain off its bond/angle minimum so every term has a force
    r = s.cartesian()
    r[:, :nchain] += rng.normal(0.0, 0.08, (3, nchain))
    sc = np.linalg.inv(s.co) @ r
    s.xp0, s.yp0, s.zp0 = sc[0], sc[1], sc[2]
    return s


def _energy(o, which):
    if which == "n0":
        _, e = o.intra_n0()
        return sum(sum(v) for v in e.values())
    _, e = o.intra_torsions()
    return sum(e)


@pytest.mark.parametrize("which", ["n0", "tors"])
def test_bonded_forces_are_minus_energy_gradient(which):
    s = chain_system()
    o = oracle.Oracle(s, nthreads=1)
    F = o.intra_n0()[0] if which == "n0" else o.intra_torsions()[0]
    assert o.last_skipped == 0
    h = 1e-6
    for a in [0, 3, 7, 12, 20, 23]:
        for ax in range(3):
            num = []
            for sgn in (1, -1):
                t = s.copy()
                cart = t.cartesian()
                cart[ax, a] += sgn * h
                sc = np.linalg.inv(t.co) @ cart
                t.xp0, t.yp0, t.zp0 = sc[0], sc[1], sc[2]
                num.append(_energy(oracle.Oracle(t, nthreads=1), which))
            fd = -(num[0] - num[1]) / (2 * h)
            scale = max(1.0, abs(F[ax, a])) * 2e-6 + 1e-9
            assert abs(fd - F[ax, a]) < scale, (which, a, ax, fd, F[ax, a])


def test_bond_and_bend_energies_closed_form():
    s = chain_system()
    s.bend_ub_k = None
    s.itors = None
    o = oracle.Oracle(s, nthreads=1)
    _, e = o.intra_n0()
    r = s.cartesian()
    ub = 0.0
    for (a, b), k, r0 in zip(s.bonds - 1, s.bond_k, s.bond_r0):
        ub += k * (np.linalg.norm(r[:, b] - r[:, a]) - r0) ** 2
    ua = 0.0
    for (a, b, c), k, t0 in zip(s.bends - 1, s.bend_k, s.bend_t0):
        u, v = r[:, a] - r[:, b], r[:, c] - r[:, b]
        th = math.acos(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v))
        ua += k * (th - t0) ** 2
    assert e["bond"][0] == pytest.approx(ub, rel=1e-12)
    assert e["bend"][0] == pytest.approx(ua, rel=1e-12)
    assert e["bond"][1] == 0.0 and e["bend"][1] == 0.0


def test_torsion_energy_is_cosine_of_dihedral():
    s = chain_system()
    o = oracle.Oracle(s, nthreads=1)
    _, (u, _) = o.intra_torsions()
    r = s.cartesian()
    ref = 0.0
    for (a, b, c, d), n, V in zip(s.tors - 1, s.tors_n, s.tors_k):
        b1, b2, b3 = r[:, b] - r[:, a], r[:, c] - r[:, b], r[:, d] - r[:, c]
        n1, n2 = np.cross(b1, b2), np.cross(b2, b3)
        phi = math.atan2(np.dot(np.cross(n1, n2), b2 / np.linalg.norm(b2)), np.dot(n1, n2))
        sig = -1.0 if n < 0 else 1.0
        ref += sig * (abs(V) - V * math.cos(abs(n) * phi))
    assert u == pytest.approx(ref, rel=1e-10)


def test_degenerate_torsion_is_skipped():
    s = chain_system()
    r = s.cartesian()
    a, b, c, d = s.tors[0] - 1
    # put atom d on the b-c axis: sin of the second bend angle vanishes
    r[:, d] = r[:, c] + (r[:, c] - r[:, b])
    sc = np.linalg.inv(s.co) @ r
    s.xp0, s.yp0, s.zp0 = sc[0], sc[1], sc[2]
    o = oracle.Oracle(s, nthreads=1)
    o.intra_torsions()
    assert o.last_skipped >= 1
