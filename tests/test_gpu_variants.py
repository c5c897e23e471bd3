"""GPU parity of the shell-kernel variants against the FP64 oracle:
force_rem (REM segment scaling), force_alchemy (soft-core alchemy) and
force_ALCHEMY_shift (the shifted potential, selected by
orac_gpu_set_alchemy_shift), plus the alchemical PME charges and work of
do_pmesh_alchemy.

Tolerances are those of the standard parity tests: forces relative RMS
<= 1e-5, energies relative <= 1e-6 of the value or of the sum of the term
magnitudes when the value cancels, stress <= 1e-5 of its norm.  dU/dlambda
from the GPU's analytic chain rule is compared with a central difference of
the oracle's U(lambda) (step 1e-4, truncation error ~1e-8 relative) at
relative 1e-5.
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
LAM = dict(ladd=0.3, lrm=0.6, laddq=0.4, lrmq=0.7)
LAM0 = dict(ladd0=0.2, lrm0=0.5, laddq0=0.35, lrmq0=0.65)
# the pair forms of the alchemy variant: soft core (force_alchemy) and
# test4's shifted potential, SHIFT-POT 4.0 0.35 (force_ALCHEMY_shift)
FORMS = {"soft": {}, "shift": dict(shifted=True, qshift=4.0, ljshift=0.35)}


def small_box():
    s = systems.water_box(nwat=64, box=16.5, lattice=4, jitter=0.25, seeds=(1, 2, 3, 4), nfft=(16, 16, 16))
    s.ncell = None
    s.shells = systems.Shells(rcutm=4.0, rtolm=0.4, rneim=0.4, rcutl=5.5, rtoll=0.4, rneil=0.4, rcuth=7.0,
                              rtolh=0.5, rneih=0.5)
    return s


@functools.lru_cache(maxsize=None)
def system(name):
    if name == "water64":
        s = small_box()
        ss = np.ones(s.ntap, np.int32)
        ss[0:9] = -2
        ss[9:15] = 2
        rem = np.zeros(s.ntap, np.uint8)
        rem[0:12] = 1
    elif name == "config1":
        s = systems.config1_water()
        ss = np.ones(s.ntap, np.int32)
        ss[0:30] = -2
        rem = np.zeros(s.ntap, np.uint8)
        rem[0:60] = 1
    elif name == "polymer_small":
        s = systems.polymer_in_water(nchain=240, nwat=900, box=32.0, nfft=(36, 36, 36), order=5, group_size=5,
                                     name="polymer_small")
        ss = np.ones(s.ntap, np.int32)
        ss[20:30] = -2  # a stretch of the chain: intramolecular exclusions matter
        rem = (s.ss_index == 1).astype(np.uint8)  # solute tempering
    else:
        raise KeyError(name)
    s.ss_alchemy = ss
    s.rematom = rem
    return s


def rel_rms(F, Fref):
    return float(np.sqrt(((F - Fref) ** 2).sum() / (Fref ** 2).sum()))


def close(g, r, scale, what):
    tol = ENERGY_REL * max(abs(r), scale, 1e-300)
    assert abs(g - r) <= tol, f"{what}: gpu {g!r} oracle {r!r} diff {g - r:.3e} tol {tol:.3e}"


def pair(name, variant, **kw):
    from orac_b200.engine import Engine

    s = system(name)
    o = oracle.Oracle(s.copy())
    g = Engine(s.copy())
    if variant == "rem":
        o.set_rem(s.rematom, kw["kind"], kw["factor"])
        g.set_rem(s.rematom, kw["kind"], kw["factor"])
    else:
        form = FORMS[kw.get("form", "soft")]
        o.set_alchemy(s.ss_alchemy, 0.5, 0.5, **form)
        g.set_alchemy(s.ss_alchemy, 0.5, 0.5, **form)
        lam = dict(kw.get("lam", LAM))
        lam.update(kw.get("lam0", {}))
        o.set_lambda(**lam)
        g.set_lambda(**lam, dlam=kw.get("dlam"))
    o.update_lists()
    g.update_lists()
    return o, g


def compare_shell(o, g, shell):
    Fr, uer, str_ = o.shell(shell)
    Fg, en, stg = g.shell(shell)
    ueg = g.ue6(en)
    assert rel_rms(Fg, Fr) <= FORCE_RMS, f"{shell}: force rel RMS {rel_rms(Fg, Fr):.3e}"
    scale = np.abs(uer).sum()
    for k in range(6):
        close(ueg[k], uer[k], 0.0, f"{shell} energy {k}")
    assert np.linalg.norm(stg - str_) <= STRESS_REL * max(np.linalg.norm(str_), 1e-300)
    return o.last_extra.copy(), g.variant_energies(), scale


@pytest.mark.parametrize("shell", ["m", "l", "h"])
@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("name", ["water64", "config1", "polymer_small"])
def test_rem_shell_parity(name, kind, shell):
    o, g = pair(name, "rem", kind=kind, factor=0.4)
    xr, xg, scale = compare_shell(o, g, shell)
    close(xg[0], xr[0], scale, f"{shell} seg_ene")


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("shell", ["m", "l", "h"])
@pytest.mark.parametrize("name", ["water64", "config1", "polymer_small"])
def test_alchemy_shell_parity(name, shell, form):
    o, g = pair(name, "alch", lam0=LAM0, form=form)
    xr, xg, scale = compare_shell(o, g, shell)
    close(xg[1], xr[1], scale, f"{shell} dwrk")
    close(xg[2], xr[2], scale, f"{shell} U0 LJ")
    close(xg[3], xr[3], scale, f"{shell} U0 Coulomb")


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("shell", ["m", "l", "h"])
@pytest.mark.parametrize("name", ["water64", "polymer_small"])
def test_alchemy_dudl_matches_oracle_central_difference(name, shell, form):
    lam = 0.4
    h = 1e-4
    o, g = pair(name, "alch", lam=dict(ladd=0.0, lrm=lam, laddq=0.0, lrmq=lam), dlam=[0.0, 1.0, 0.0, 1.0], form=form)
    g.shell(shell)
    dudl = g.variant_energies()[4]
    u = []
    for sgn in (1, -1):
        l2 = lam + sgn * h
        o.set_lambda(ladd=0.0, lrm=l2, laddq=0.0, lrmq=l2)
        o.update_lists()
        _, ue, _ = o.shell(shell)
        u.append(ue.sum())
    fd = (u[0] - u[1]) / (2 * h)
    assert abs(dudl - fd) <= 1e-5 * max(abs(fd), 1e-12), (dudl, fd)
    assert dudl != 0.0


@pytest.mark.parametrize("name", ["water64", "polymer_small"])
def test_alchemy_pme_charges_and_work(name):
    o, g = pair(name, "alch", lam0=LAM0)
    s = system(name)
    lq = np.where(s.ss_alchemy == 2, LAM["laddq"], np.where(s.ss_alchemy == -2, -LAM["lrmq"], 0.0))
    lq0 = np.where(s.ss_alchemy == 2, LAM0["laddq0"], np.where(s.ss_alchemy == -2, -LAM0["lrmq0"], 0.0))
    t = s.copy()
    t.charge = (1.0 - np.abs(lq)) * s.charge
    Fr, er, sr = oracle.Oracle(t).fft_pme()
    t0 = s.copy()
    t0.charge = (1.0 - np.abs(lq0)) * s.charge
    _, er0, _ = oracle.Oracle(t0).fft_pme()
    Fg, eg, sg = g.fft_pme()
    assert rel_rms(Fg, Fr) <= FORCE_RMS
    close(eg, er, 0.0, "eer")
    assert np.linalg.norm(sg - sr) <= STRESS_REL * np.linalg.norm(sr)
    close(g.variant_energies()[5], er - er0, abs(er), "PME work")


def test_alchemy_pme_dudl_matches_oracle_central_difference():
    from orac_b200.engine import Engine

    s = system("polymer_small")
    lam, h = 0.4, 1e-4
    g = Engine(s.copy())
    g.set_alchemy(s.ss_alchemy)
    g.set_lambda(0.0, lam, 0.0, lam, dlam=[0.0, 1.0, 0.0, 1.0])
    g.fft_pme()
    dudl = g.variant_energies()[6]
    e = []
    for sgn in (1, -1):
        t = s.copy()
        lq = np.where(s.ss_alchemy == -2, lam + sgn * h, 0.0)
        t.charge = (1.0 - lq) * s.charge
        e.append(oracle.Oracle(t).fft_pme()[1])
    fd = (e[0] - e[1]) / (2 * h)
    assert abs(dudl - fd) <= 1e-5 * abs(fd), (dudl, fd)


@pytest.mark.parametrize("form", sorted(FORMS))
def test_md_window_dudl_is_derivative_of_potential(form):
    """Record column 15 of an alchemical MD window (shells, SPME, erf
    corrections, self term, and ORAC's intra-alchemical corrections:
    fnb14_alchemy's 1-4 pairs and ferrf_alchemy_add over listqq) against the
    central difference of the oracle's potential energy at the same
    configuration (a 1e-9 fs step leaves the atoms in place), with either
    pair form."""
    from orac_b200.engine import Engine

    s = systems.ligand_in_water()
    lam, h = 0.3, 1e-4
    g = Engine(s.copy())
    g.set_alchemy(s.ss_alchemy, **FORMS[form])
    g.set_lambda(0.0, lam, 0.0, lam, dlam=[0.0, 1.0, 0.0, 1.0])
    g.md_setup(1e-9, 2, 4, 6, "l")
    rec = g.md_run(1, energy_every=1)
    dudl = rec[0, 15]
    a = s.intra_lists()
    u = []
    for sgn in (1, -1):
        lr = lam + sgn * h
        o = oracle.Oracle(s.copy())
        o.set_alchemy(s.ss_alchemy, **FORMS[form])
        o.set_lambda(0.0, lr, 0.0, lr)
        o.update_lists()
        esh = sum(o.shell(sh)[1].sum() for sh in "mlh")
        t = s.copy()
        t.charge = np.where(s.ss_alchemy == -2, 1.0 - lr, 1.0) * s.charge
        ot = oracle.Oracle(t)
        epme = ot.fft_pme()[1]
        eerf = 0.0
        for pairs, fudge, iz in ((a["lbnd"], 1.0, 1), (t.constraints.ravel(), 1.0, 0), (a["int13"], 1.0, 1),
                                 (a["int14"], 1.0 - s.fudge, 1)):
            if len(pairs):
                eerf += ot.ferrf(np.asarray(pairs).reshape(-1, 2), fudge, iz=iz)[1].sum()
        eself = ot.cself()[0]
        lam_at = o.alch_lambdas(s.ss_alchemy, 0.0, lr)
        e14 = o.fnb14_alchemy(lam_at, lam_at)[1].sum()
        eqq = o.ferrf_alchemy_add(o.alch_listqq(s.ss_alchemy), lam_at)[1].sum()
        u.append(esh + epme + eerf + eself + e14 + eqq)
    fd = (u[0] - u[1]) / (2 * h)
    assert abs(dudl - fd) <= 1e-5 * abs(fd), (dudl, fd)


def test_lambda_change_after_md_setup_reaches_the_step_graphs():
    """A window moved to a new lambda after md_setup: its next step reports
    the dU/dlambda of a window set up at that lambda directly (the captured
    step graphs are captured again when a parameter changes; 1e-9 fs steps
    leave the atoms in place)."""
    from orac_b200.engine import Engine

    s = systems.ligand_in_water()

    def window(lam):
        g = Engine(s.copy())
        g.set_alchemy(s.ss_alchemy)
        g.set_lambda(0.0, lam, 0.0, lam, dlam=[0.0, 1.0, 0.0, 1.0])
        g.md_setup(1e-9, 2, 4, 6, "l")
        return g

    g = window(0.2)
    d_a = g.md_run(1, energy_every=1)[0, 15]
    g.set_lambda(0.0, 0.7, 0.0, 0.7, dlam=[0.0, 1.0, 0.0, 1.0])
    d_b = g.md_run(1, energy_every=1)[0, 15]
    g.close()
    ref = window(0.7)
    ref.md_run(1, energy_every=1)
    d_ref = ref.md_run(1, energy_every=1)[0, 15]
    ref.close()
    assert abs(d_b - d_a) > 1e-3 * abs(d_a)
    assert abs(d_b - d_ref) <= 1e-6 * abs(d_ref), (d_b, d_ref)


def test_intra_alchemical_corrections_energies_match_oracle():
    """ORAC's intra-alchemical corrections in an alchemical MD window at
    lambda 0.45: record column 13 (1-4 and intra-group pairs, fnb14_alchemy
    for the 1-4 pairs) and column 14 (erf corrections of the scaled charges
    plus ferrf_alchemy_add over listqq) against the oracle's restatements at
    the same configuration (1e-9 fs step), relative 1e-9 (both FP64)."""
    from orac_b200.engine import Engine

    s = systems.ligand_in_water()
    lam = 0.45
    g = Engine(s.copy())
    g.set_alchemy(s.ss_alchemy)
    g.set_lambda(0.0, lam, 0.0, lam, dlam=[0.0, 1.0, 0.0, 1.0])
    g.md_setup(1e-9, 2, 4, 6, "l")
    rec = g.md_run(1, energy_every=1)[0]
    g.close()
    o = oracle.Oracle(s.copy())
    lam_at = o.alch_lambdas(s.ss_alchemy, 0.0, lam)
    e14 = o.fnb14_alchemy(lam_at, lam_at)[1].sum() + o.fnbgrp()[1].sum()
    assert abs(rec[13] - e14) <= 1e-9 * abs(e14), (rec[13], e14)
    a = s.intra_lists()
    t = s.copy()
    t.charge = np.where(s.ss_alchemy == -2, 1.0 - lam, 1.0) * s.charge
    ot = oracle.Oracle(t)
    eerf = 0.0
    for pairs, fudge, iz in ((a["lbnd"], 1.0, 1), (t.constraints.ravel(), 1.0, 0), (a["int13"], 1.0, 1),
                             (a["int14"], 1.0 - s.fudge, 1)):
        if len(pairs):
            eerf += ot.ferrf(np.asarray(pairs).reshape(-1, 2), fudge, iz=iz)[1].sum()
    lst = o.alch_listqq(s.ss_alchemy)
    assert len(lst) > 500
    eqq = o.ferrf_alchemy_add(lst, lam_at)[1].sum()
    assert abs(rec[14] - (eerf + eqq)) <= 1e-9 * (abs(eerf) + abs(eqq)), (rec[14], eerf, eqq)
