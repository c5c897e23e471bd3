"""GPU parity of ORAC's Nose-Hoover thermostats (THERMOS, NVT) against the
FP64 oracle's restatement of the M-level sequence (src/mtsmd.f:2556-2618,
2932, 3109-3170): the thermostats' coordinates and velocities, every
energy term with the extended system's total, and the positions, step by
step, on three molecular layouts: a flexible chain (one unconstrained
molecule with bonded levels) in rigid water, a 40-atom ligand in rigid
water, and FKBP12 with its ligand and bonds to hydrogen rigid (constraint
clusters inside large molecules); a batch of thermostatted systems moves
each one as it moves alone."""
import numpy as np
import pytest

import oracle
from orac_b200 import systems
from orac_b200.engine import Batch, Engine
from orac_b200.lib import OracGpuError

pytestmark = pytest.mark.gpu

SCHED = dict(dt_h=4.0, lrespa=2, mrespa=4, nupdte=1000, rshk="l", n1respa=2, n0respa=2)
# energies and thermostat velocities to 1e-5 relative (FP32 forces summed in
# fixed point against FP64; the thermostats integrate the kinetic energy's
# excess, which the trajectories' 1e-7 A differences move at that level)
RTOL = 1e-5


def chain():
    return systems.polymer_in_water(nchain=60, nwat=600, box=28.0, nfft=(32, 32, 32), order=4, group_size=3,
                                    name="chain60")


def econst(s):
    a, b = oracle.Oracle(s).cself()
    return a + b


def pair(s, sched, nu, temp=300.0):
    ec = econst(s)
    g = Engine(s.copy())
    g.set_thermostat(temp, *nu)
    g.md_setup(sched["dt_h"], sched["lrespa"], sched["mrespa"], sched["nupdte"], sched["rshk"],
               n1respa=sched["n1respa"], n0respa=sched["n0respa"], econst=ec)
    o = oracle.OracleMD(s.copy(), sched["dt_h"], sched["lrespa"], sched["mrespa"], sched["nupdte"], sched["rshk"],
                        n1respa=sched["n1respa"], n0respa=sched["n0respa"], econst=ec)
    o.set_thermostat(temp, *nu)
    return g, o


def compare(g, o, steps, xtol=1e-6):
    for step in range(steps):
        rg = g.md_run(1, energy_every=1)
        ro = o.run(1, energy_every=1)
        for k in list(range(1, 11)) + [12, 13, 14, 15]:
            np.testing.assert_allclose(rg[:, k], ro[:, k], rtol=RTOL, atol=1e-9,
                                       err_msg=f"record column {k} after step {step}")
        eg, pg, qg, ng, _ = g.md_thermostat()
        eo, po, qo, no, _ = o.thermostat()
        assert list(ng) == list(no)
        np.testing.assert_allclose(qg, qo, rtol=1e-14)
        # a thermostat whose velocity crosses zero is compared on the scale
        # of the largest one
        np.testing.assert_allclose(pg, po, rtol=RTOL, atol=RTOL * np.abs(po).max(), err_msg=f"etap after step {step}")
        np.testing.assert_allclose(eg, eo, rtol=RTOL, atol=RTOL * np.abs(eo).max(), err_msg=f"eta after step {step}")
    xg, _ = g.md_state()
    xo, _ = o.state()
    assert np.abs(xg - xo).max() < xtol
    return pg


def test_nvt_chain_in_water_matches_the_oracle():
    """Stiff thermostats (100 cm^-1) on the hot lattice start: the
    thermostats move at once, every one in the same direction as the
    oracle's."""
    g, o = pair(chain(), SCHED, (100.0, 100.0, 100.0))
    etap = compare(g, o, 8)
    assert (etap > 1e-4).all()
    g.close()
    o.close()


def test_nvt_ligand_in_water_matches_the_oracle():
    g, o = pair(systems.ligand_in_water(), SCHED, (20.0, 20.0, 20.0))
    compare(g, o, 5)
    g.close()
    o.close()


def test_nvt_f0_matches_the_oracle():
    """FKBP12 and its ligand in water from test2's restart (ORAC's F0 at
    300 K), test4's r-RESPA and THERMOS frequencies (20 cm^-1)."""
    from test_oracle_ne import F0_MD, f0_test4

    s = f0_test4(1)
    g, o = pair(s, F0_MD, (20.0, 20.0, 20.0))
    compare(g, o, 2)
    g.close()
    o.close()


def test_nvt_batch_moves_each_system_as_alone():
    base = chain()
    walkers = []
    for k in range(3):
        s = base.copy()
        rng = np.random.default_rng(200 + k)
        scale = 1.0 + 0.05 * rng.standard_normal(s.ntap)
        s.vx, s.vy, s.vz = s.vx * scale, s.vy * scale, s.vz * scale
        walkers.append(s)

    def make(s):
        g = Engine(s.copy())
        g.set_thermostat(300.0, 50.0, 50.0, 50.0)
        g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                   n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
        return g

    alone = []
    for s in walkers:
        g = make(s)
        g.md_run(6)
        alone.append((g.md_state()[0], g.md_thermostat()))
        g.close()
    engines = [make(s) for s in walkers]
    b = Batch(engines)
    b.run(6)
    b.close()
    for k, g in enumerate(engines):
        x, _ = g.md_state()
        th = g.md_thermostat()
        assert np.array_equal(x, alone[k][0]), k
        assert np.array_equal(th[1], alone[k][1][1]) and np.array_equal(th[0], alone[k][1][0]), k
        g.close()
    assert len({round(a[1][1][2], 12) for a in alone}) == 3  # the walkers' thermostats differ


def test_thermostat_setter_errors():
    s = chain()
    g = Engine(s.copy())
    with pytest.raises(OracGpuError):
        g.set_thermostat(300.0, 0.0, 10.0, 10.0)
    g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"])
    with pytest.raises(OracGpuError):
        g.set_thermostat(300.0, 10.0, 10.0, 10.0)  # after md_setup
    with pytest.raises(OracGpuError):
        g.md_thermostat()  # NVE: no thermostats
    g.close()


def test_nvt_restart_continues_the_run(tmp_path):
    """An ORAC restart file of a thermostatted run (positions, velocities, the
    hoover records gh = eta, vh = etap) written after 4 steps and read into a
    new context continues the run: 4 + 3 steps against 7 in one go (the
    restarted context builds its lists again; the pair set and the
    fixed-point forces are the same)."""
    from test_oracle_nvt import restored

    from orac_b200 import oracio

    s = chain()

    def make(sys_):
        g = Engine(sys_)
        g.set_thermostat(300.0, 50.0, 50.0, 50.0)
        g.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"],
                   n1respa=SCHED["n1respa"], n0respa=SCHED["n0respa"])
        return g

    a = make(s.copy())
    a.md_run(4)
    x, v = a.md_state()
    eta, etap, _, _, _ = a.md_thermostat()
    p = str(tmp_path / "nvt.rst")
    oracio.write_rst(p, s.co, x, v, nstep=4, temp=300.0, thermostat=(eta, etap))
    a.md_run(3)
    r = oracio.read_rst(p, s.ntap)
    b = make(restored(s, r["xyz"], r["v"]))
    b.set_thermostat_state(r["eta"], r["etap"])
    b.md_run(3)
    xa, _ = a.md_state()
    xb, _ = b.md_state()
    assert np.abs(xa - xb).max() < 1e-8
    np.testing.assert_allclose(b.md_thermostat()[1], a.md_thermostat()[1], rtol=1e-8)
    a.close()
    b.close()


def test_nvt_ne_f0_from_orac_thermostat_state_matches_the_oracle():
    """test4's walker 1 on ORAC's system: the non-equilibrium schedule with
    test4's THERMOS (300 K, 20 cm^-1) started from the thermostats' state of
    ORAC's restart file; the GPU's work, lambdas and thermostats against the
    oracle's after each of 4 outer steps (60 fs)."""
    import os

    from test_oracle_ne import F0_FORM, F0_MD, f0_test4

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    d = np.load(os.path.join(here, "ne_test4.npz"))
    r = np.load(os.path.join(here, "f0_orac_records.npz"))
    sched = d["schedule"]
    args = (sched[:, 0] * 1000.0, sched[:, 1], sched[:, 2], sched[:, 3], sched[:, 4])
    s = f0_test4(0)
    g = Engine(s.copy())
    g.set_alchemy(s.ss_alchemy, 0.5, 0.5, **F0_FORM)
    g.set_lambda(0.0, 0.0, 0.0, 0.0)
    g.set_schedule(*args)
    g.set_thermostat(300.0, 20.0, 20.0, 20.0)
    g.md_setup(F0_MD["dt_h"], F0_MD["lrespa"], F0_MD["mrespa"], F0_MD["nupdte"], F0_MD["rshk"],
               n1respa=F0_MD["n1respa"], n0respa=F0_MD["n0respa"])
    g.set_thermostat_state(r["eta0"], r["etap0"])
    o = oracle.OracleMD(s.copy(), F0_MD["dt_h"], F0_MD["lrespa"], F0_MD["mrespa"], F0_MD["nupdte"], F0_MD["rshk"],
                        n1respa=F0_MD["n1respa"], n0respa=F0_MD["n0respa"])
    o.set_alchemy(s.ss_alchemy, [0.0] * 8, **F0_FORM)
    o.set_schedule(*args)
    o.set_thermostat(300.0, 20.0, 20.0, 20.0)
    o.set_thermostat_state(r["eta0"], r["etap0"])
    for step in range(4):
        g.md_run(1)
        o.run(1)
        wg, tg, lg, _ = g.md_work()
        wo, to, lo, _ = o.work()
        assert tg == to and lg == lo
        np.testing.assert_allclose(wg, wo, rtol=1e-5, atol=1e-8, err_msg=f"work after step {step}")
        pg, po = g.md_thermostat()[1], o.thermostat()[1]
        np.testing.assert_allclose(pg, po, rtol=RTOL, atol=RTOL * np.abs(po).max(), err_msg=f"etap after step {step}")
    g.close()
    o.close()
