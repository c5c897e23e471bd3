"""GPU r-RESPA driver against the CPU oracle's restatement of ORAC's loop.

Tolerances: the first steps of the two trajectories agree in every energy
term to 1e-5 relative and in positions to 1e-6 A (FP32 forces with
fixed-point sums vs FP64; the trajectories separate later, as any two MD
codes do); total energy stays within 0.5% of the kinetic energy over 100
steps of the liquid-density box; replaying captured graphs gives bitwise
the same state as launching every kernel directly (fixed-point force sums
do not depend on the order of the atomics).
"""
import numpy as np
import pytest

import oracle
from orac_b200 import systems
from orac_b200.engine import Engine

pytestmark = pytest.mark.gpu

SCHED = dict(dt_h=4.0, lrespa=2, mrespa=4, nupdte=6, rshk="l")


def econst(s):
    a, b = oracle.Oracle(s).cself()
    return a + b


def test_md_first_steps_match_oracle():
    s = systems.config1_liquid()
    ec = econst(s)
    g = Engine(s.copy())
    g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"], econst=ec)
    rg = g.md_run(3, energy_every=1)
    o = oracle.OracleMD(s.copy(), SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                        econst=ec)
    ro = o.run(3, energy_every=1)
    for k in list(range(1, 11)) + [12, 13, 14]:
        np.testing.assert_allclose(rg[:, k], ro[:, k], rtol=1e-5, atol=1e-9, err_msg=f"record column {k}")
    xg, _ = g.md_state()
    xo, _ = o.state()
    assert np.abs(xg - xo).max() < 1e-6


def test_md_energy_conservation_liquid():
    s = systems.config1_liquid()
    g = Engine(s)
    g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"], econst=econst(s))
    g.md_run(20)  # let the lattice start relax
    rec = g.md_run(100, energy_every=5)
    etot = rec[:, 10]
    ekin = rec[:, 1]
    assert np.isfinite(etot).all()
    assert (etot.max() - etot.min()) < 5e-3 * ekin.mean(), (etot.min(), etot.max(), ekin.mean())


def test_md_graph_replay_is_bitwise_direct_launch():
    s = systems.config1_water()
    states = []
    for graphs in (True, False):
        g = Engine(s.copy())
        g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"], graphs=graphs)
        g.md_run(8)
        states.append(g.md_state())
        g.close()
    assert np.array_equal(states[0][0], states[1][0])
    assert np.array_equal(states[0][1], states[1][1])


def test_md_energy_records_leave_the_trajectory_unchanged():
    """Steps that also evaluate energies apply the same forces as steps that
    do not, to FP32 rounding (the switching function of the forces is the
    FP32 one in both; the FP64 one enters the energies only): positions
    agree to 1e-6 A after 12 steps."""
    s = chain_box()
    states = []
    for every in (0, 3):
        g = Engine(s.copy())
        g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"])
        g.md_run(12, energy_every=every)
        states.append(g.md_state())
        g.close()
    assert np.abs(states[0][0] - states[1][0]).max() < 1e-6


def chain_box():
    return systems.polymer_in_water(nchain=60, nwat=600, box=28.0, nfft=(32, 32, 32), order=4, group_size=3,
                                    name="chain60")


@pytest.mark.parametrize("n1respa,n0respa", [(1, 1), (2, 2)])
def test_md_flexible_chain_matches_oracle(n1respa, n0respa):
    """Bonded N0 (bonds, bends) and N1 (torsions, 1-4) levels, the erf
    corrections at the reciprocal level, and the n1respa/n0respa loops."""
    s = chain_box()
    ec = econst(s)
    g = Engine(s.copy())
    g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"], n1respa=n1respa,
               n0respa=n0respa, econst=ec)
    rg = g.md_run(3, energy_every=1)
    o = oracle.OracleMD(s.copy(), SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                        econst=ec, n1respa=n1respa, n0respa=n0respa)
    ro = o.run(3, energy_every=1)
    for k in list(range(1, 11)) + [12, 13, 14]:
        np.testing.assert_allclose(rg[:, k], ro[:, k], rtol=1e-5, atol=1e-9, err_msg=f"record column {k}")
    xg, _ = g.md_state()
    xo, _ = o.state()
    assert np.abs(xg - xo).max() < 1e-6
    assert rg[0, 12] != 0.0 and rg[0, 13] != 0.0


def test_md_flexible_chain_energy_conservation():
    s = chain_box()
    g = Engine(s)
    g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"], econst=econst(s))
    g.md_run(10)
    rec = g.md_run(100, energy_every=5)
    etot, ekin = rec[:, 10], rec[:, 1]
    assert np.isfinite(etot).all()
    assert (etot.max() - etot.min()) < 5e-3 * ekin.mean(), (etot.min(), etot.max(), ekin.mean())


def _drift(rec):
    """Total-energy drift (kJ/mol per ps, least squares) and the RMS of the
    residual about that line, of energy records of 4-fs steps."""
    from orac_b200 import units

    t = rec[:, 0] * 4.0e-3
    e = rec[:, 10] * units.KJMOL
    p = np.polyfit(t, e, 1)
    return float(p[0]), float(np.std(e - np.polyval(p, t)))


def test_energy_conservation_over_1000_steps_matches_the_oracle():
    """1,000 outer steps (4 ps) of the liquid box from its seeded start, NVE:
    the GPU's total-energy drift and fluctuation against the FP64 oracle's
    over the same run (tests/golden/liquid_drift_oracle.npz, made by
    tests/golden/make_drift.py).  The trajectories separate after a few
    hundred steps, so the two are compared as statistics: drift within
    3 kJ/mol/ps of the oracle's (the total is about 4.3e4 kJ/mol), residual
    fluctuation within a factor 2."""
    import os

    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "liquid_drift_oracle.npz"))
    s = systems.config1_liquid()
    g = Engine(s.copy())
    g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"], econst=econst(s))
    rec = g.md_run(int(ref["nsteps"]), energy_every=int(ref["every"]))
    g.close()
    assert np.all(rec[:, 11] == 0)
    d_g, f_g = _drift(rec)
    d_o, f_o = _drift(ref["rec"])
    assert abs(d_g - d_o) <= 3.0, (d_g, d_o)
    assert 0.5 * f_o <= f_g <= 2.0 * f_o, (f_g, f_o)
