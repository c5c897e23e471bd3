"""Checks of the oracle's REM (force_rem) and soft-core alchemy
(force_alchemy) variants of the shell kernel, on the CPU.

Pinned by properties the reference's formulas imply:
  - alchemy with every lambda 0 (all atoms fully on, no soft core) is the
    standard force; REM with rem_factor 1 is the standard force;
  - forces are minus the gradient of the energy the variant defines
    (alchemy: U(lambda); REM: E - (1 - s) seg_ene, because selected pairs
    are scaled by s in the force but reported unscaled);
  - the REM force is linear in rem_factor, and seg_ene(either) =
    seg_ene(both) + seg_ene(exactly one);
  - dwrk = U(lambda) - U(lambda0) (src/force_alchemy.f:683-688);
  - the same for the shifted potential (force_ALCHEMY_shift), which at
    every lambda 0 is the standard force too and elsewhere differs from the
    soft core.
"""
import numpy as np
import pytest

import oracle
from orac_b200 import systems


def small_water(seed=0):
    s = systems.water_box(nwat=64, box=16.5, lattice=4, jitter=0.25, seeds=(seed + 1, seed + 2, seed + 3, seed + 4),
                          nfft=(16, 16, 16))
    s.ncell = None
    s.shells = systems.Shells(rcutm=4.0, rtolm=0.4, rneim=0.4, rcutl=5.5, rtoll=0.4, rneil=0.4, rcuth=7.0,
                              rtolh=0.5, rneih=0.5)
    return s


def alch_water(seed=0, added=True):
    s = small_water(seed)
    ss = np.ones(s.ntap, np.int32)
    ss[0:9] = -2  # three removed waters
    if added:
        ss[9:15] = 2  # two added waters
    s.ss_alchemy = ss
    return s


def rem_water(seed=0):
    s = small_water(seed)
    rem = np.zeros(s.ntap, np.uint8)
    rem[0:12] = 1  # a four-water segment
    s.rematom = rem
    return s


LAM = dict(ladd=0.3, lrm=0.6, laddq=0.4, lrmq=0.7)


SHIFT = dict(shifted=True, qshift=4.0, ljshift=0.35)  # test4's SHIFT-POT 4.0 0.35


def _oracle(s, variant=None, lam=None, lam0=None, rem=None):
    o = oracle.Oracle(s, nthreads=2)
    if variant in ("alch", "shift"):
        o.set_alchemy(s.ss_alchemy, 0.5, 0.5, **(SHIFT if variant == "shift" else {}))
        lam = lam or dict(ladd=0.0, lrm=0.0, laddq=0.0, lrmq=0.0)
        kw = dict(lam)
        if lam0:
            kw.update({k + "0": v for k, v in lam0.items()})
        o.set_lambda(**kw)
    elif variant == "rem":
        o.set_rem(s.rematom, *rem)
    o.update_lists()
    return o


def _rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def test_alch_set_tables():
    t = oracle.alch_set(0.25, 0.5)
    assert t[:, 2 + 4].tolist() == [0.0, 1.0]
    assert t[:, 3 + 4].tolist() == [0.25, 0.75]
    assert t[:, -1 + 4].tolist() == [0.5, 0.5]
    assert t[:, 4 + 4].tolist() == [0.0, 1.0] and t[:, -4 + 4].tolist() == [0.0, 1.0]
    assert t[:, 0 + 4].tolist() == [0.0, 0.0]
    q = oracle.alch_set(0.25, 0.5, intramol=True, qq=True)
    assert q[:, 4 + 4].tolist() == [0.0625, 0.9375] and q[:, -4 + 4].tolist() == [0.25, 0.75]
    lj = oracle.alch_set(0.25, 0.5, intramol=True, ljintra=False)
    assert lj[:, 4 + 4].tolist() == [0.25, 0.75]


@pytest.mark.parametrize("shell", ["m", "l", "h"])
def test_alchemy_at_zero_lambda_is_the_standard_force(shell):
    """Removed atoms only: removed-added pairs (class 0) never interact.
    The two kernels agree to ~1e-8, not to rounding: ORAC derives the
    soft-core sigma with 2**(1./6.) taken in single precision
    (src/mtsmd.f:1298), the LJ tables with a double 2**(1/6) (covnb)."""
    s = alch_water(added=False)
    Fs, us, ss = _oracle(s).shell(shell)
    o = _oracle(s, "alch")
    Fa, ua, sa = o.shell(shell)
    assert _rel(Fa, Fs) < 1e-7
    assert np.allclose(ua, us, rtol=1e-7, atol=1e-9 * np.abs(us).sum())
    assert np.allclose(sa, ss, rtol=1e-7, atol=1e-8 * np.abs(ss).max())
    assert abs(o.last_extra[1]) < 1e-12 * np.abs(ua).sum()


@pytest.mark.parametrize("shell", ["m", "l", "h"])
def test_rem_with_unit_factor_is_the_standard_force(shell):
    s = rem_water()
    Fs, us, ss = _oracle(s).shell(shell)
    Fr, ur, sr = _oracle(s, "rem", rem=(0, 1.0)).shell(shell)
    assert np.array_equal(Fr, Fs) and np.array_equal(ur, us) and np.array_equal(sr, ss)


def _fd_check(s, make, energy, atoms, h=1e-6, tol=2e-6):
    o = make(s)
    F, ue, _ = o.shell_eval
    for a in atoms:
        for ax in range(3):
            num = []
            for sgn in (1, -1):
                t = s.copy()
                cart = t.cartesian()
                cart[ax, a] += sgn * h
                sc = np.linalg.inv(t.co) @ cart
                t.xp0, t.yp0, t.zp0 = sc[0], sc[1], sc[2]
                num.append(energy(make(t)))
            fd = -(num[0] - num[1]) / (2 * h)
            assert abs(fd - F[ax, a]) < tol * max(1.0, abs(F[ax, a])) + 1e-7, (a, ax, fd, F[ax, a])


@pytest.mark.parametrize("shell", ["m", "h"])
def test_alchemy_forces_are_minus_energy_gradient(shell):
    s = alch_water()

    def make(t):
        o = _oracle(t, "alch", lam=LAM)
        o.shell_eval = o.shell(shell)
        return o

    atoms = [0, 1, 5, 10, 13, 40]  # removed, added and normal atoms
    _fd_check(s, make, lambda o: o.shell_eval[1].sum(), atoms)


@pytest.mark.parametrize("shell", ["m", "h"])
def test_rem_forces_are_minus_scaled_energy_gradient(shell):
    s = rem_water()
    fac = 0.4

    def make(t):
        o = _oracle(t, "rem", rem=(0, fac))
        o.shell_eval = o.shell(shell)
        return o

    def energy(o):
        return o.shell_eval[1].sum() - (1.0 - fac) * o.last_extra[0]

    _fd_check(s, make, energy, [0, 4, 11, 12, 30, 50])


def test_rem_force_is_linear_in_factor_and_energy_unscaled():
    s = rem_water()
    out = {}
    for f in (0.0, 1.0, 0.35):
        o = _oracle(s, "rem", rem=(0, f))
        out[f] = o.shell("l") + (o.last_extra.copy(),)
    F0, F1, Fx = out[0.0][0], out[1.0][0], out[0.35][0]
    assert _rel(Fx, F0 + 0.35 * (F1 - F0)) < 1e-12
    assert np.allclose(out[0.35][1], out[1.0][1], rtol=1e-13, atol=0)
    assert out[0.35][3][0] == pytest.approx(out[1.0][3][0], rel=1e-13)


def test_rem_segment_kinds_partition_the_pairs():
    s = rem_water()
    seg = {}
    for kind in (0, 1, 2):
        o = _oracle(s, "rem", rem=(kind, 0.5))
        o.shell("m")
        seg[kind] = o.last_extra[0]
    assert seg[0] == pytest.approx(seg[1] + seg[2], rel=1e-12)
    assert seg[1] != 0.0 and seg[2] != 0.0


def test_rem_whole_system_segment_energy_is_the_total():
    s = rem_water()
    s.rematom = np.ones(s.ntap, np.uint8)
    o = _oracle(s, "rem", rem=(0, 0.5))
    F, ue, _ = o.shell("m")
    assert o.last_extra[0] == pytest.approx(ue.sum(), rel=1e-12)
    Fs, _, _ = _oracle(s).shell("m")
    assert _rel(F, 0.5 * Fs) < 1e-13


def test_alchemy_work_is_energy_difference():
    s = alch_water()
    lam0 = dict(ladd=0.2, lrm=0.5, laddq=0.35, lrmq=0.65)
    o = _oracle(s, "alch", lam=LAM, lam0=lam0)
    _, ue, _ = o.shell("m")
    dwrk, c0, q0 = o.last_extra[1], o.last_extra[2], o.last_extra[3]
    _, ue_l, _ = _oracle(s, "alch", lam=LAM).shell("m")
    _, ue_0, _ = _oracle(s, "alch", lam=lam0).shell("m")
    assert np.allclose(ue, ue_l, rtol=1e-14)
    assert dwrk == pytest.approx(ue_l.sum() - ue_0.sum(), rel=1e-10)
    assert c0 + q0 == pytest.approx(ue_0.sum(), rel=1e-10)
    assert dwrk != 0.0


def test_alchemy_fully_removed_atoms_do_not_interact():
    """lrm = lrmq = 1: removed atoms have scale 0 against normal atoms, and
    pairs removed-added have scale 0 at any lambda, so the removed waters
    only feel each other (scale 1 among themselves): by Newton's third law
    their net force vanishes."""
    s = alch_water()
    o = _oracle(s, "alch", lam=dict(ladd=0.0, lrm=1.0, laddq=0.0, lrmq=1.0))
    F, ue, _ = o.shell("m")
    Fm = F[:, :9].sum(axis=1)
    assert np.allclose(Fm, 0.0, atol=1e-12 * np.abs(F).max())
    assert np.abs(F[:, :9]).max() > 0.0


@pytest.mark.parametrize("shell", ["m", "l", "h"])
def test_shifted_at_zero_lambda_is_the_standard_force(shell):
    """Removed atoms only, as for the soft core (removed-added pairs never
    interact); with no shift left the kernels agree to the sigma factor's
    single-precision 2**(1./6.)."""
    s = alch_water(added=False)
    F0, ue0, st0 = _oracle(s).shell(shell)
    F1, ue1, st1 = _oracle(s, "shift").shell(shell)
    assert _rel(F1, F0) < 1e-6
    assert np.allclose(ue1, ue0, rtol=1e-6, atol=1e-9 * np.abs(ue0).max())


@pytest.mark.parametrize("shell", ["m", "h"])
def test_shifted_forces_are_minus_energy_gradient(shell):
    s = alch_water()

    def make(t):
        o = _oracle(t, "shift", lam=LAM)
        o.shell_eval = o.shell(shell)
        return o

    _fd_check(s, make, lambda o: o.shell_eval[1].sum(), [0, 1, 5, 10, 13, 40])


def test_shifted_work_is_energy_difference_and_differs_from_the_soft_core():
    s = alch_water()
    lam0 = dict(ladd=0.2, lrm=0.5, laddq=0.35, lrmq=0.65)
    o = _oracle(s, "shift", lam=LAM, lam0=lam0)
    F, ue, _ = o.shell("m")
    dwrk = o.last_extra[1]
    _, ue_0, _ = _oracle(s, "shift", lam=lam0).shell("m")
    assert dwrk == pytest.approx(ue.sum() - ue_0.sum(), rel=1e-10)
    Fs, ues, _ = _oracle(s, "alch", lam=LAM).shell("m")
    assert _rel(F, Fs) > 1e-3 and abs(ue.sum() - ues.sum()) > 1e-6 * abs(ues.sum())
