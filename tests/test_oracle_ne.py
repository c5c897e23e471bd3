"""The oracle's non-equilibrium alchemy loop (ORAC's steered alchemy):
alchemic (src/alchemic.f) pinned on the lambdas ORAC printed in test4's
four work files (tests/golden/ne_test4.npz), and the bookkeeping of the
lambda update and the work (src/mtsmd.f:2963-2999, 3042-3044) on the
40-atom ligand in the liquid box."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from orac_b200 import systems

HERE = os.path.dirname(os.path.abspath(__file__))
SCHED = dict(dt_h=4.0, lrespa=2, mrespa=4, nupdte=1000, rshk="l", n1respa=2, n0respa=2)


def alchemic(sched_ps, t_fs):
    L = oracle.lib()
    D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    L.orc_alchemic.argtypes = [C.c_int, D, D, D, D, D, C.c_double, D]
    cols = [np.ascontiguousarray(sched_ps[:, k], dtype=np.float64) for k in range(5)]
    cols[0] = cols[0] * 1000.0  # ORAC reads the times in ps and keeps fs (src/read_potential.f:756)
    g = np.zeros(4)
    L.orc_alchemic(len(cols[0]), *cols, float(t_fs), g)
    return g


def test_alchemic_matches_the_lambdas_orac_printed_in_test4():
    """print_alchemic_wrk (src/print_alchemic_work.f) writes 1 - ladd,
    1 - laddq, lrm, lrmq at rtime / 1000 ps: every row of the four walkers'
    1.5.wrk against the restatement at the row's time, to the printed
    digits."""
    d = np.load(os.path.join(HERE, "golden", "ne_test4.npz"))
    sched = d["schedule"]
    for k in range(1, 5):
        for row in d[f"wrk{k}"]:
            g = alchemic(sched, row[0] * 1000.0)
            printed = row[1:5]
            mine = np.array([1.0 - g[0], 1.0 - g[2], g[1], g[3]])
            np.testing.assert_allclose(mine, printed, rtol=0, atol=6e-6, err_msg=f"walker {k} t={row[0]} ps")


def test_alchemic_edges():
    sched = np.array([[0.0, 0.0, 0.0, 0.0, 0.0], [0.1, 0.5, 0.2, 0.3, 0.4], [0.2, 1.0, 1.0, 1.0, 1.0]])
    # before the first point: ladd = laddq = 1, lrm = lrmq = 0
    np.testing.assert_array_equal(alchemic(sched, -1.0), [1.0, 0.0, 1.0, 0.0])
    # on a shared point the later slice wins (its start value)
    np.testing.assert_allclose(alchemic(sched, 100.0), [0.5, 0.3, 0.2, 0.4], rtol=0, atol=1e-15)
    # linear inside a slice; the last point's values after the end
    np.testing.assert_allclose(alchemic(sched, 50.0), [0.25, 0.15, 0.1, 0.2], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(alchemic(sched, 500.0), [1.0, 1.0, 1.0, 1.0])


def ne_md(s, times, lams, nsteps):
    o = oracle.OracleMD(s.copy(), SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                        n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
    o.set_alchemy(s.ss_alchemy, [0.0] * 8)
    o.set_schedule(times, *lams)
    out = []
    for _ in range(nsteps):
        o.run(1)
        out.append(o.work())
    o.close()
    return out


@pytest.fixture(scope="module")
def ligand():
    return systems.ligand_in_water()


def test_a_schedule_that_holds_the_lambdas_does_no_work(ligand):
    """lambda = lambda0 throughout: every term's U(lambda) - U(lambda0) is
    zero to the last bit."""
    lams = ([1.0, 1.0], [1.0, 1.0], [0.3, 0.3], [0.6, 0.6])
    for w, rtime, g, terms in ne_md(ligand, [0.0, 400.0], lams, 2):
        assert w == 0.0 and not terms.any(), (w, terms)
        np.testing.assert_allclose(g, [1.0, 0.3, 1.0, 0.6], rtol=0, atol=1e-15)


def test_lambdas_follow_the_schedule_and_work_accumulates(ligand):
    """Charges off over 40 fs: rtime advances one outer step (4 fs) per step,
    the lambdas are alchemic's at rtime, and removing the ligand's charges
    costs work in every M step (the electrostatic terms dominate)."""
    times = [0.0, 40.0, 80.0]
    lams = ([1.0, 1.0, 1.0], [1.0, 1.0, 1.0], [0.0, 0.0, 1.0], [0.0, 1.0, 1.0])
    sched = np.array([[t / 1000.0, a, aq, r, rq] for t, a, aq, r, rq in zip(times, *lams)])
    res = ne_md(ligand, times, lams, 3)
    prev = 0.0
    for k, (w, rtime, g, terms) in enumerate(res):
        assert abs(rtime - 4.0 * (k + 1)) < 1e-12
        np.testing.assert_allclose(g, alchemic(sched, rtime), rtol=0, atol=1e-15)
        assert w != prev and terms[1] != 0.0  # the held L-shell term moved too
        prev = w


# ORAC's test4 on F0: the FKBP12 ligand (atoms 1-52, DEFINE_ALCHEMICAL_ATOM
# 1 52 off) switched off along 15.off with the shifted potential (SHIFT-POT
# 4.0 0.35), test4's shells (5.0/8.1/12.5 A, tolerances 0.3, margins
# 0.5/0.5/1.5), SPME alpha 0.37 on 48 x 49 x 48 order 4, r-RESPA
# 15/3/1.5/0.75/0.375 fs, bonds to hydrogen rigid, lists every 60 fs; the
# walkers start from test2's restart files ij4i0000 (PAR0001), ij4i0001
# (PAR0002) and ij4i0003 (PAR0004)
F0_WALKERS = {0: 1, 1: 2, 2: 4}  # f0_orac_records state -> test4 walker


def f0_test4(k):
    from orac_b200 import oracio

    gold = os.path.join(HERE, "golden")
    tp, rst = oracio.split_arrays(dict(np.load(os.path.join(gold, "f0_fkbp12.npz"))))
    if k > 0:
        r = np.load(os.path.join(gold, "f0_orac_records.npz"))
        rst = dict(rst, co=r[f"co{k}"], xyz=r[f"xyz{k}"], v=r[f"v{k}"])
    sh = systems.Shells(rcutm=5.0, rtolm=0.3, rneim=0.5, rcutl=8.1, rtoll=0.3, rneil=0.5, rcuth=12.5, rtolh=0.3,
                        rneih=1.5)
    s = oracio.system_from_orac(tp, rst, alphal=0.37, nfft=(48, 49, 48), order=4, shells=sh, ncell=(18, 18, 18),
                                fudge=0.83333, lj_fudge=0.5, name=f"F0_test4_{k}", rigid_hydrogen=True)
    ss = np.ones(s.ntap, np.int32)
    ss[:52] = -2
    s.ss_alchemy = ss
    return s


F0_MD = dict(dt_h=15.0, lrespa=5, mrespa=2, nupdte=4, rshk="l", n1respa=2, n0respa=2)
F0_FORM = dict(shifted=True, qshift=4.0, ljshift=0.35)


@pytest.mark.parametrize("k", sorted(F0_WALKERS))
def test_f0_test4_work_at_60_fs_matches_what_orac_printed(k):
    """The restatement's work after 60 fs (4 outer steps, 40 M steps) of
    test4's schedule against the first line of the walker's 1.5.wrk.  ORAC
    ran NPT with Nose-Hoover thermostats and a ligand-target COM restraint;
    this run is NVE without the restraint: the two agree to 0.4% (0.2-0.33%
    below ORAC for the three walkers)."""
    from orac_b200 import units

    d = np.load(os.path.join(HERE, "golden", "ne_test4.npz"))
    sched = d["schedule"]
    s = f0_test4(k)
    o = oracle.OracleMD(s.copy(), F0_MD["dt_h"], F0_MD["lrespa"], F0_MD["mrespa"], F0_MD["nupdte"], F0_MD["rshk"],
                        n1respa=F0_MD["n1respa"], n0respa=F0_MD["n0respa"])
    o.set_alchemy(s.ss_alchemy, [0.0] * 8, **F0_FORM)
    o.set_schedule(sched[:, 0] * 1000.0, sched[:, 1], sched[:, 2], sched[:, 3], sched[:, 4])
    o.run(4)
    w, rtime, g, _ = o.work()
    o.close()
    row = d[f"wrk{F0_WALKERS[k]}"][0]
    assert abs(rtime - 1000.0 * row[0]) < 1e-9
    np.testing.assert_allclose([1.0 - g[0], 1.0 - g[2], g[1], g[3]], row[1:5], rtol=0, atol=6e-6)
    np.testing.assert_allclose(w * units.KJMOL, row[5], rtol=4e-3)
