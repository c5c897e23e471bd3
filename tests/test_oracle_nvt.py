"""The oracle's Nose-Hoover thermostats (ORAC's THERMOS at the M level,
src/mtsmd.f:2556-2618, 2932, 3109-3170): degrees of freedom and masses as
find_thermos and cov_thermos set them, the NVE limit of a massive
thermostat, and the extended system's conserved energy while stiff
thermostats pull a hot box down (the thermostats' energy grows by
thousands of times the drift)."""
import numpy as np
import pytest

import oracle
from orac_b200 import systems, units

SCHED = dict(dt_h=4.0, lrespa=2, mrespa=4, nupdte=1000, rshk="l", n1respa=2, n0respa=2)


@pytest.fixture(scope="module")
def chain():
    # 60 flexible chain atoms (solute: one unconstrained molecule with bonded
    # N0/N1 levels) in 600 rigid waters (solvent); the lattice start is hot
    return systems.polymer_in_water(nchain=60, nwat=600, box=28.0, nfft=(32, 32, 32), order=4, group_size=3,
                                    name="chain60")


def md(s, nu=None, steps=40, every=5):
    o = oracle.OracleMD(s.copy(), SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                        n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
    if nu is not None:
        o.set_thermostat(300.0, nu, nu, nu)
    rec = o.run(steps, energy_every=every)
    out = (rec, o.state(), o.thermostat() if nu is not None else None)
    o.close()
    return out


def test_degrees_of_freedom_and_masses(chain):
    """find_thermos: 3 per molecule (centres of mass), 3 per atom less 3 per
    molecule less the constraints (solute, solvent); cov_thermos:
    Q = 2 ndf k T / (2 pi c nu)^2 in amu A^2."""
    o = oracle.OracleMD(chain.copy(), SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"],
                        SCHED["rshk"])
    o.set_thermostat(300.0, 10.0, 20.0, 40.0)
    eta, etap, q, ndf, e = o.thermostat()
    o.close()
    assert list(ndf) == [3 * 601, 3 * 60 - 3, 3 * 1800 - 3 * 600 - 1800]
    om = 2.0 * np.pi * 2.997925e10 * np.array([10.0, 20.0, 40.0])
    want = 2.0 * ndf * units.BOLTZ * 300.0 / om ** 2 / (units.UNITM * units.UNITL ** 2)
    np.testing.assert_allclose(q, want, rtol=1e-14)
    assert not eta.any() and not etap.any() and e == 0.0


def test_a_massive_thermostat_leaves_the_nve_trajectory(chain):
    """nu -> 0 makes Q huge and etap ~ 0: the run is NVE's to rounding."""
    r0, (x0, v0), _ = md(chain, None, steps=10)
    r1, (x1, v1), th = md(chain, 1e-4, steps=10)
    assert np.abs(x1 - x0).max() < 1e-9
    np.testing.assert_allclose(r1[:, 1], r0[:, 1], rtol=1e-9)
    assert np.abs(th[1]).max() < 1e-12


def test_stiff_thermostats_cool_the_box_and_conserve_the_extended_energy(chain):
    """nu = 100 cm^-1 (a 333 fs period) at 300 K on a start near 1,400 K:
    within 160 fs the kinetic energy falls to a fifth; the thermostats take
    up the difference (their energy rises by several internal units) while
    the extended system's total (column 10) moves by less than the NVE
    run's total does over the same steps, give or take 2e-4 units."""
    rn, _, _ = md(chain, None)
    rt, _, th = md(chain, 100.0)
    assert rt[-1, 1] < 0.2 * rt[0, 1]
    assert th[4] > 1.0 and rt[-1, 15] == th[4]
    dn = np.abs(rn[:, 10] - rn[0, 10]).max()
    dt = np.abs(rt[:, 10] - rt[0, 10]).max()
    assert dt < dn + 2e-4, (dt, dn)
    assert (th[0] > 0).all() and (th[1] > 0).all()  # a hot box: every thermostat pulls


def restored(s, x, v):
    """The system at a restart's positions (Cartesian, 3 x N) and velocities."""
    r = s.copy()
    sc = np.linalg.solve(r.co, x)
    r.xp0, r.yp0, r.zp0 = sc[0].copy(), sc[1].copy(), sc[2].copy()
    r.xyz_restart = x.copy()
    r.vx, r.vy, r.vz = v[0].copy(), v[1].copy(), v[2].copy()
    return r


def test_restart_with_the_thermostat_state_continues_the_run(chain):
    """Positions, velocities and ORAC's thermostat records of a restart
    (src/readrs.f:247-251) continue the run: 4 + 3 steps against 7 in one go."""
    def make(s):
        o = oracle.OracleMD(s, SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                            n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
        o.set_thermostat(300.0, 50.0, 50.0, 50.0)
        return o

    a = make(chain.copy())
    a.run(4)
    x, v = a.state()
    eta, etap, _, _, _ = a.thermostat()
    a.run(3)
    b = make(restored(chain, x, v))
    b.set_thermostat_state(eta, etap)
    b.run(3)
    xa, _ = a.state()
    xb, _ = b.state()
    assert np.abs(xa - xb).max() < 1e-8
    np.testing.assert_allclose(b.thermostat()[1], a.thermostat()[1], rtol=1e-8)
    a.close()
    b.close()


def test_f0_test4_with_the_restart_thermostats_matches_what_orac_printed():
    """test4's walker 1 on ORAC's system with test4's THERMOS (300 K, 20
    cm^-1) started from the thermostats' state ORAC wrote into its restart
    (tests/golden/f0_orac_records.npz: eta, etap of test2's ij4i0000.rst):
    the work after 60 fs against the first line of ORAC's 1.5.wrk (ORAC's
    run adds the barostat and a COM restraint: 0.4%, as the NVE run)."""
    import os

    from test_oracle_ne import F0_FORM, F0_MD, F0_WALKERS, f0_test4

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    d = np.load(os.path.join(here, "ne_test4.npz"))
    r = np.load(os.path.join(here, "f0_orac_records.npz"))
    sched = d["schedule"]
    s = f0_test4(0)
    o = oracle.OracleMD(s.copy(), F0_MD["dt_h"], F0_MD["lrespa"], F0_MD["mrespa"], F0_MD["nupdte"], F0_MD["rshk"],
                        n1respa=F0_MD["n1respa"], n0respa=F0_MD["n0respa"])
    o.set_alchemy(s.ss_alchemy, [0.0] * 8, **F0_FORM)
    o.set_schedule(sched[:, 0] * 1000.0, sched[:, 1], sched[:, 2], sched[:, 3], sched[:, 4])
    o.set_thermostat(300.0, 20.0, 20.0, 20.0)
    o.set_thermostat_state(r["eta0"], r["etap0"])
    o.run(4)
    w = o.work()[0]
    eta, etap, _, _, _ = o.thermostat()
    o.close()
    np.testing.assert_allclose(w * units.KJMOL, d[f"wrk{F0_WALKERS[0]}"][0, 5], rtol=4e-3)
    assert np.all(eta != r["eta0"])  # the thermostats moved from ORAC's state
