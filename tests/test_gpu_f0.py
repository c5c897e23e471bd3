"""The real ORAC system F0 on the GPU against the FP64 oracle.

F0 is the solvated FKBP12-ligand system of the reference's tests as ORAC
itself assembled it (its topology-parameter file) at a state ORAC wrote (a
restart file at step 30): 14,900 atoms, 1,715 of them protein and ligand,
5,082 charge groups of up to four atoms, 90 LJ types, 4,500 1-4 pairs,
5,732 proper and 339 improper torsions (tests/golden/f0_fkbp12.npz, made by
tests/golden/make_f0.py, read by orac_b200.oracio).  The parameters are
those of the reference's test1 input: SPME alpha 0.37 on 48^3 with order 4,
shells 5.1/7.8/10.0 A with tolerances 0.3 A and neighbour margins
0.4/0.5/1.5 A, 18^3 linked cells, 1-4 fudge 0.83333 (Coulomb) and 0.5
(LJ), r-RESPA 15/3/1.5/0.75/0.375 fs.  Every bond is flexible in the
force tests; the constrained MD test makes the bonds to hydrogen rigid
(test1's STRETCHING HEAVY: 14,041 constraints, the protein's through the
iterative SHAKE/RATTLE of large molecules, the waters' by SETTLE).

Tolerances as in the other parity tests: forces relative RMS <= 1e-5,
energies <= 1e-6 relative (of the value or of the sum of the shell's term
magnitudes where the value cancels), stress <= 1e-5 of its norm; FP64
bonded terms to 1e-10; two MD steps (160 inner steps) agree with the
oracle's in every energy column to 1e-5 relative and in positions to
1e-6 A; so do two constrained steps.
"""
import functools
import os

import numpy as np
import pytest

import oracle
from orac_b200 import oracio, systems

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "f0_fkbp12.npz")


@functools.lru_cache(maxsize=None)
def f0(rigid_hydrogen=False):
    tp, rst = oracio.split_arrays(dict(np.load(FIX)))
    sh = systems.Shells(rcutm=5.1, rtolm=0.3, rneim=0.4, rcutl=7.8, rtoll=0.3, rneil=0.5, rcuth=10.0, rtolh=0.3,
                        rneih=1.5)
    return oracio.system_from_orac(tp, rst, alphal=0.37, nfft=(48, 48, 48), order=4, shells=sh, ncell=(18, 18, 18),
                                   fudge=0.83333, lj_fudge=0.5, name="F0_fkbp12", rigid_hydrogen=rigid_hydrogen)


def rel_rms(F, Fref):
    return float(np.sqrt(((F - Fref) ** 2).sum() / (Fref ** 2).sum()))


@pytest.fixture(scope="module")
def pair():
    from orac_b200.engine import Engine

    s = f0()
    o = oracle.Oracle(s.copy())
    g = Engine(s.copy())
    o.update_lists()
    g.update_lists()
    yield o, g
    g.close()


@pytest.mark.parametrize("shell", ["m", "l", "h"])
def test_f0_shell_parity(pair, shell):
    o, g = pair
    Fr, uer, sr = o.shell(shell)
    Fg, en, sg = g.shell(shell)
    ueg = g.ue6(en)
    assert rel_rms(Fg, Fr) <= 1e-5, rel_rms(Fg, Fr)
    scale = np.abs(uer).sum()
    for k in range(6):
        assert abs(ueg[k] - uer[k]) <= 1e-6 * max(abs(uer[k]), 1e-300) or abs(ueg[k] - uer[k]) <= 1e-7 * scale, \
            (k, ueg[k], uer[k])
    assert np.linalg.norm(sg - sr) <= 1e-5 * np.linalg.norm(sr)


def test_f0_pme_parity(pair):
    o, g = pair
    Fr, er, sr = o.fft_pme()
    Fg, eg, sg = g.fft_pme()
    assert rel_rms(Fg, Fr) <= 1e-5
    assert abs(eg - er) <= 1e-6 * abs(er)
    assert np.linalg.norm(sg - sr) <= 1e-5 * np.linalg.norm(sr)


def test_f0_intramolecular_parity(pair):
    o, g = pair
    Fr, er = o.intra_n0()
    Fg, eg = g.intra_n0()
    assert rel_rms(Fg, Fr) <= 1e-10
    ref = [er["bond"][0], er["bond"][1], er["bend"][0], er["bend"][1], er["itors"][0], er["itors"][1]]
    np.testing.assert_allclose(eg, ref, rtol=1e-10, atol=1e-300)
    Ft, et = o.intra_torsions()
    F14, e14 = o.fnb14()
    Fgp, egp = o.fnbgrp()
    Fg1, eg1 = g.intra_n1()
    assert rel_rms(Fg1, Ft + F14 + Fgp) <= 1e-10
    np.testing.assert_allclose(eg1[:2], et, rtol=1e-10)
    np.testing.assert_allclose(eg1[2:6], e14, rtol=1e-10, atol=1e-300)


def test_f0_bonded_energies_equal_orac_printed_record():
    """The CUDA bonded levels at F0's state against the energy record ORAC
    printed for it (test2/PAR0001/out0001 line 818, kept in
    tests/golden/f0_orac_records.npz), with bonds to hydrogen rigid as in
    that run: stretching, bending, improper and proper torsion energies equal
    the printed two decimals."""
    from orac_b200 import units
    from orac_b200.engine import Engine

    rec = np.load(os.path.join(os.path.dirname(FIX), "f0_orac_records.npz"))
    p = dict(zip([str(k) for k in rec["keys"]], rec["printed"][0]))
    g = Engine(f0(True).copy())
    _, e0 = g.intra_n0()
    _, e1 = g.intra_n1()
    g.close()
    K = units.KJMOL
    got = {"SltStr": e0[0] * K, "SltBen": e0[2] * K, "SltItor": e0[4] * K, "SltPtor": e1[0] * K}
    for col, v in got.items():
        assert abs(v - p[col]) <= 0.006, (col, v, p[col])


@pytest.mark.parametrize("rigid", [False, True])
def test_f0_md_steps_match_oracle(rigid):
    from orac_b200.engine import Engine

    s = f0(rigid)
    a, b = oracle.Oracle(s.copy()).cself()
    sched = (15.0, 5, 2, 6, "l")
    g = Engine(s.copy())
    g.md_setup(*sched, n1respa=2, n0respa=2, econst=a + b)
    rg = g.md_run(2, energy_every=1)
    o = oracle.OracleMD(s.copy(), *sched, econst=a + b, n1respa=2, n0respa=2)
    ro = o.run(2, energy_every=1)
    for k in list(range(1, 11)) + [12, 13, 14]:
        np.testing.assert_allclose(rg[:, k], ro[:, k], rtol=1e-5, atol=1e-9, err_msg=f"record column {k}")
    xg, _ = g.md_state()
    xo, _ = o.state()
    assert np.abs(xg - xo).max() < 1e-6, np.abs(xg - xo).max()
    g.close()
