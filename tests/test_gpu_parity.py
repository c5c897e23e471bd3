"""GPU parity: liborac_gpu.so through its C ABI against the FP64 CPU oracle
on identical inputs.

Tolerances (stated for every comparison):
  forces   relative RMS  sqrt(sum|F-Fref|^2 / sum|Fref|^2) <= 1e-5
           (ORAC's own check_force metric, src/pme_code.f:378-396)
  energies relative error <= 1e-6 of the oracle's value, or 1e-6 of the
           sum of the term's magnitudes when the value itself cancels
  stress   <= 1e-5 of the oracle tensor's Frobenius norm
  lists    the number of group pairs in every shell list is identical
"""
import functools

import numpy as np
import pytest

import oracle
from orac_b200 import systems

pytestmark = pytest.mark.gpu

FORCE_RMS = 1e-5
ENERGY_REL = 1e-6
STRESS_REL = 1e-5


def small_box(nw=64, box=16.5, seed=0):
    s = systems.water_box(nwat=nw, box=box, lattice=4, jitter=0.25, seeds=(seed + 1, seed + 2, seed + 3, seed + 4),
                          nfft=(16, 16, 16))
    s.ncell = None
    s.shells = systems.Shells(rcutm=4.0, rtolm=0.4, rneim=0.4, rcutl=5.5, rtoll=0.4, rneil=0.4, rcuth=7.0,
                              rtolh=0.5, rneih=0.5)
    s.name = "water64"
    return s


def pair_across_face():
    s = systems.two_waters(sep=(3.2, 0.4, -0.3), box=20.0, across_face=True)
    s.ncell = None
    s.shells = systems.Shells(rcutm=2.5, rtolm=0.5, rneim=0.4, rcutl=3.3, rtoll=0.4, rneil=0.4, rcuth=6.0,
                              rtolh=0.5, rneih=0.5)
    return s


def polymer_small():
    s = systems.polymer_in_water(nchain=240, nwat=900, box=32.0, nfft=(36, 36, 36), order=5, group_size=5,
                                 name="polymer_small")
    return s


@functools.lru_cache(maxsize=None)
def system(name):
    if name == "pair_face":
        return pair_across_face()
    if name == "water64":
        return small_box()
    if name == "config1":
        return systems.config1_water()
    if name == "polymer_small":
        return polymer_small()
    if name == "config2":
        return systems.config2_polymer()
    raise KeyError(name)


@functools.lru_cache(maxsize=None)
def engines(name):
    from orac_b200.engine import Engine

    s = system(name)
    o = oracle.Oracle(s.copy())
    g = Engine(s.copy())
    o.update_lists()
    g.update_lists()
    return o, g


def rel_rms(F, Fref):
    den = (Fref ** 2).sum()
    if den == 0:
        return float(np.sqrt((F ** 2).sum()))
    return float(np.sqrt(((F - Fref) ** 2).sum() / den))


def assert_energy(g, r, scale, what):
    tol = ENERGY_REL * max(abs(r), scale, 1e-300)
    assert abs(g - r) <= tol, f"{what}: gpu {g!r} oracle {r!r} diff {g - r:.3e} tol {tol:.3e}"


SYSTEMS = ["pair_face", "water64", "config1", "polymer_small", "config2"]


@pytest.mark.parametrize("name", SYSTEMS)
def test_list_sizes_match_oracle(name):
    o, g = engines(name)
    pairs, _ = g.list_pairs()
    ng = o.s.ngrp
    for sh in "hlm":
        assert pairs[sh] == len(o.lists[sh]) - ng, (sh, pairs[sh], len(o.lists[sh]) - ng)


@pytest.mark.parametrize("shell", ["m", "l", "h"])
@pytest.mark.parametrize("name", SYSTEMS)
def test_shell_parity(name, shell):
    o, g = engines(name)
    Fr, uer, str_ = o.shell(shell)
    Fg, en, stg = g.shell(shell)
    ueg = g.ue6(en)
    assert rel_rms(Fg, Fr) <= FORCE_RMS, f"force rel RMS {rel_rms(Fg, Fr):.3e}"
    for k, lab in enumerate(["LJ slt", "LJ slv", "LJ mixed", "Coul slt", "Coul slv", "Coul mixed"]):
        assert_energy(ueg[k], uer[k], 0.0, f"{shell} {lab}")
    nrm = np.linalg.norm(str_)
    assert np.linalg.norm(stg - str_) <= STRESS_REL * max(nrm, 1e-300), (stg, str_)
    assert en["virs"] == 0.0 and en["virsp"] == 0.0
    # list refresh of the next inner shell matches too
    pairs, _ = g.list_pairs()
    nxt = {"h": "l", "l": "m"}.get(shell)
    if nxt:
        assert pairs[nxt] == len(o.lists[nxt]) - o.s.ngrp


@pytest.mark.parametrize("name", ["water64", "config1", "polymer_small", "config2"])
def test_pme_parity(name):
    o, g = engines(name)
    Fr, er, sr = o.fft_pme()
    Fg, eg, sg = g.fft_pme()
    assert rel_rms(Fg, Fr) <= FORCE_RMS, f"force rel RMS {rel_rms(Fg, Fr):.3e}"
    assert_energy(eg, er, 0.0, "eer")
    assert np.linalg.norm(sg - sr) <= STRESS_REL * np.linalg.norm(sr), (sg, sr)


@pytest.mark.parametrize("dims,order", [((32, 32, 32), 4), ((36, 30, 28), 5), ((45, 40, 42), 6), ((20, 20, 20), 8)])
def test_do_pmesh_kspace_grids(dims, order):
    """Odd orders, odd and mixed-radix grid sizes (2, 3, 5, 7)."""
    s = system("water64")
    o, g = engines("water64")
    r = s.cartesian()
    recip = 0.5 * np.linalg.inv(s.co).T
    Fr, er, vr = o.do_pmesh_kspace(r[0], r[1], r[2], s.charge, recip, s.volume, 0.35, order, dims)
    Fg, eg, vg = g.do_pmesh_kspace(r[0], r[1], r[2], s.charge, recip, s.volume, 0.35, order, dims)
    assert rel_rms(Fg, Fr) <= FORCE_RMS
    assert_energy(eg, er, 0.0, "eer")
    assert np.linalg.norm(vg - vr) <= STRESS_REL * np.linalg.norm(vr)


def test_fnb14_ferrf_cself_parity():
    o, g = engines("polymer_small")
    Fr, ur = o.fnb14()
    Fg, ug = g.fnb14()
    assert rel_rms(Fg, Fr) <= FORCE_RMS
    for k in range(4):
        assert_energy(ug[k], ur[k], 0.0, f"fnb14[{k}]")
    s = o.s
    for pairs, fudge in ((s.bonds, 1.0), (s.bend13, 1.0), (s.int14, 1.0 - s.fudge)):
        Fr, fr = o.ferrf(pairs, fudge)
        Fg, fg = g.ferrf(pairs, fudge)
        assert rel_rms(Fg, Fr) <= FORCE_RMS
        for k in range(2):
            assert_energy(fg[k], fr[k], 0.0, "ferrf")
        # iz = 0: energy only (constraints at start-up, src/mtsmd.f:1641-1645)
        F0, f0 = g.ferrf(pairs, fudge, iz=0)
        assert not F0.any()
    a, b = o.cself()
    c, d = g.cself()
    assert_energy(c, a, 0.0, "self slt")
    assert_energy(d, b, 0.0, "self slv")


def test_fnbgrp_parity():
    o, g = engines("polymer_small")
    assert len(o.s.ingrp) > 0
    Fr, ur = o.fnbgrp()
    Fg, ug = g.fnbgrp()
    assert rel_rms(Fg, Fr) <= FORCE_RMS
    for k in range(4):
        assert_energy(ug[k], ur[k], 0.0, f"fnbgrp[{k}]")
