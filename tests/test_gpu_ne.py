"""GPU parity of a non-equilibrium alchemical run (ORAC's steered alchemy,
the NE work swarms of test3/test4) against the FP64 oracle's NE loop: the
lambdas follow a schedule on the device, moved before every M shell
(src/alchemic.f, src/mtsmd.f:2963-2999), and the work adds ORAC's terms
(src/mtsmd.f:3042-3044).  The 40-atom ligand in the liquid box loses its
charges over 40 fs, then its LJ over the next 40, in the order of test3's
and test4's schedule (15.off: charges first); both pair forms (soft core,
and test4's shifted potential).  Every outer step the lambdas and rtime
agree exactly, the work within the tolerance below, and the trajectory
stays on the oracle's."""
import os

import numpy as np
import pytest

import oracle
from orac_b200 import systems
from orac_b200.engine import Batch, Engine

pytestmark = pytest.mark.gpu

SCHED = dict(dt_h=4.0, lrespa=2, mrespa=4, nupdte=1000, rshk="l", n1respa=2, n0respa=2)
TIMES = [0.0, 40.0, 80.0]
LAMS = dict(ladded=[1.0, 1.0, 1.0], laddedq=[1.0, 1.0, 1.0], lremoved=[0.0, 0.0, 1.0], lremovedq=[0.0, 1.0, 1.0])
FORMS = {"soft": {}, "shift": dict(shifted=True, qshift=4.0, ljshift=0.35)}
# work (ORAC's internal energy unit, 1e4 kJ/mol): the trajectory leaves
# the FP64 one by ~1e-7 A per step, and the reciprocal term comes from FP32
# FFTs (summed as a cross term of the two transformed grids, not as the
# difference of two energies); the work follows to an absolute 1e-8 units
# (1e-4 kJ/mol) or 1e-5 of its value
WORK_RTOL, WORK_ATOL = 1e-5, 1e-8


def pair(form, s=None):
    s = systems.ligand_in_water() if s is None else s
    g = Engine(s.copy())
    g.set_alchemy(s.ss_alchemy, 0.5, 0.5, **FORMS[form])
    g.set_lambda(0.0, 0.0, 0.0, 0.0)
    g.set_schedule(TIMES, LAMS["ladded"], LAMS["laddedq"], LAMS["lremoved"], LAMS["lremovedq"])
    g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
               n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
    o = oracle.OracleMD(s.copy(), SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                        n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
    o.set_alchemy(s.ss_alchemy, [0.0] * 8, **FORMS[form])
    o.set_schedule(TIMES, LAMS["ladded"], LAMS["laddedq"], LAMS["lremoved"], LAMS["lremovedq"])
    return s, g, o


@pytest.mark.parametrize("form", ["soft", "shift"])
def test_ne_work_and_trajectory_match_the_oracle(form):
    s, g, o = pair(form)
    works = []
    for step in range(24):  # 96 fs: both stages and a stretch past the schedule's end
        g.md_run(1)
        o.run(1)
        wg, tg, lg, dg = g.md_work()
        wo, to, lo, do = o.work()
        assert tg == to, (step, tg, to)
        assert lg == lo, (step, lg, lo)
        np.testing.assert_allclose(wg, wo, rtol=WORK_RTOL, atol=WORK_ATOL,
                                   err_msg=f"work after step {step}; terms GPU - oracle {dg - do}")
        np.testing.assert_allclose(dg, do, rtol=1e-4, atol=WORK_ATOL, err_msg=f"work terms after step {step}: {dg - do}")
        works.append(wo)
    # the charges and the LJ came off: work was done (tens of kJ/mol in
    # each stage), and it stops once the schedule has ended and the held
    # terms have been evaluated again
    assert abs(works[9]) > 1e-3 and abs(works[19] - works[9]) > 1e-3
    assert works[23] == works[21]
    xg, _ = g.md_state()
    xo, _ = o.state()
    assert np.abs(xg - xo).max() < 1e-4
    # one record per M step: 8 per outer step, rtime advancing by 0.5 fs
    tr, n = g.md_work_trace()
    assert n == 24 * 8
    np.testing.assert_allclose(np.diff(tr[:, 0]), 0.5, rtol=0, atol=1e-12)
    assert tr[-1, 1] == wg
    # an energy step's record carries the work in column 15
    rec = g.md_run(1, energy_every=1)
    assert rec[0, 15] == g.md_work()[0]


def test_ne_swarm_in_one_batch_matches_each_alone():
    """A swarm of NE trajectories from different starting velocities, as
    test3/test4's MPI walkers, advanced by one graph launch per step: each
    walker's state equals its run alone bitwise (fixed-point forces), its
    work to 1e-9 (FP64 work sums in atomics of a varying order)."""
    base = systems.ligand_in_water()
    walkers = []
    for k in range(3):
        s = base.copy()
        rng = np.random.default_rng(100 + k)
        scale = 1.0 + 0.02 * rng.standard_normal(s.ntap)
        s.vx, s.vy, s.vz = s.vx * scale, s.vy * scale, s.vz * scale
        walkers.append(s)

    def make(s):
        g = Engine(s.copy())
        g.set_alchemy(s.ss_alchemy, 0.5, 0.5)
        g.set_lambda(0.0, 0.0, 0.0, 0.0)
        g.set_schedule(TIMES, LAMS["ladded"], LAMS["laddedq"], LAMS["lremoved"], LAMS["lremovedq"])
        g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                   n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
        return g

    alone = []
    for s in walkers:
        g = make(s)
        g.md_run(12)
        alone.append((g.md_work()[0], g.md_state()[0]))
        g.close()
    engines = [make(s) for s in walkers]
    b = Batch(engines)
    b.run(12)
    b.close()
    for k, g in enumerate(engines):
        w = g.md_work()[0]
        x, _ = g.md_state()
        assert abs(w - alone[k][0]) <= 1e-9 * abs(alone[k][0]), (k, w, alone[k][0])
        assert np.array_equal(x, alone[k][1]), k
        g.close()
    assert len({round(a[0], 6) for a in alone}) == 3  # the walkers differ


def test_f0_test4_work_matches_the_oracle_and_what_orac_printed():
    """test4 on the reference's own system (tests/test_oracle_ne.py has the
    setup): the GPU's work over 60 fs against the oracle's and against the
    first line of walker 1's 1.5.wrk (ORAC ran NPT with a COM restraint,
    this run NVE without it: 0.4%)."""
    from test_oracle_ne import F0_FORM, F0_MD, f0_test4

    from orac_b200 import units

    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ne_test4.npz"))
    sched = d["schedule"]
    s = f0_test4(0)
    args = (sched[:, 0] * 1000.0, sched[:, 1], sched[:, 2], sched[:, 3], sched[:, 4])
    g = Engine(s.copy())
    g.set_alchemy(s.ss_alchemy, 0.5, 0.5, **F0_FORM)
    g.set_lambda(0.0, 0.0, 0.0, 0.0)
    g.set_schedule(*args)
    g.md_setup(F0_MD["dt_h"], F0_MD["lrespa"], F0_MD["mrespa"], F0_MD["nupdte"], F0_MD["rshk"],
               n1respa=F0_MD["n1respa"], n0respa=F0_MD["n0respa"])
    o = oracle.OracleMD(s.copy(), F0_MD["dt_h"], F0_MD["lrespa"], F0_MD["mrespa"], F0_MD["nupdte"], F0_MD["rshk"],
                        n1respa=F0_MD["n1respa"], n0respa=F0_MD["n0respa"])
    o.set_alchemy(s.ss_alchemy, [0.0] * 8, **F0_FORM)
    o.set_schedule(*args)
    for step in range(4):
        g.md_run(1)
        o.run(1)
        wg, tg, lg, _ = g.md_work()
        wo, to, lo, _ = o.work()
        assert tg == to and lg == lo
        np.testing.assert_allclose(wg, wo, rtol=WORK_RTOL, atol=WORK_ATOL, err_msg=f"F0 work after step {step}")
    np.testing.assert_allclose(wg * units.KJMOL, d["wrk1"][0, 5], rtol=4e-3)
    g.close()
    o.close()
