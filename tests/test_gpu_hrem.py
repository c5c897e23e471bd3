"""Replica exchange on the GPU: rem_factor(3) lives in device memory, so a
factor rewritten between steps (orac_gpu_set_rem_factor_async, what an
exchange does) reaches the captured step graphs without capturing them
again -- bitwise the trajectory of a context whose factor was set by
orac_gpu_set_rem (which captures again); an HREM batch of four replicas
records each replica's segment energy on the device, keeps the ensembles a
permutation, swaps every attempted pair when the test is forced to accept,
and runs twice to the same states."""
import numpy as np
import pytest

from orac_b200 import hrem, systems, units
from orac_b200.engine import Engine

pytestmark = pytest.mark.gpu

SCHED = dict(dt_h=4.0, lrespa=2, mrespa=4, nupdte=6, rshk="l")
KT_300 = units.BOLTZ * 300.0 / units.UNITE  # kT at 300 K, internal units


def system():
    return systems.solvated_chains(3000, 77, solute_frac=0.08, name="hrem3000")


def engine(s, factor):
    e = Engine(s.copy())
    e.set_rem(s.rematom, 0, factor)
    e.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"])
    return e


def test_factor_rewritten_on_the_device_reaches_the_step_graphs():
    s = system()
    a = engine(s, 1.0)
    a.md_run(4)
    a.set_rem(s.rematom, 0, 0.55)  # a parameter change: the graphs are captured again
    a.md_run(4)
    xa, va = a.md_state()
    a.close()
    b = engine(s, 1.0)
    b.md_run(4)
    b.set_rem_factor_async(0.55)  # in stream order, same graphs
    b.md_run(4)
    xb, vb = b.md_state()
    b.close()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    c = engine(s, 1.0)
    c.md_run(8)
    xc, _ = c.md_state()
    c.close()
    assert not np.array_equal(xa, xc)  # the factor did change the forces


def _run(kT, intervals=5, every=3, seed=3):
    s = system()
    ladder = hrem.ladder_geometric(4, 0.5)
    engines = [engine(s, f) for f in ladder]
    h = hrem.HremBatch(engines, ladder, kT, seed=seed)
    pots, enss = [], []
    for _ in range(intervals):
        pots.append(h.interval(every))
        enss.append(h.ens.copy())
    states = [e.md_state() for e in engines]
    acc = h.acceptance()
    h.close()
    for e in engines:
        e.close()
    return pots, enss, states, acc


def test_hrem_batch_exchanges():
    pots, enss, states, acc = _run(KT_300)
    for p, ens in zip(pots, enss):
        assert np.all(np.isfinite(p)) and np.all(p != 0.0)
        assert sorted(ens.tolist()) == [0, 1, 2, 3]
    assert np.all((acc >= 0.0) & (acc <= 1.0))
    pots2, enss2, states2, _ = _run(KT_300)
    for a, b in zip(enss, enss2):
        assert np.array_equal(a, b)
    for (x, v), (x2, v2) in zip(states, states2):
        assert np.array_equal(x, x2) and np.array_equal(v, v2)


def test_hrem_forced_acceptance_swaps_every_attempted_pair():
    _, enss, _, acc = _run(1e300, intervals=4)
    # ORAC's parity (0-based ensembles): exchange step 1 pairs (1, 2),
    # step 2 pairs (0, 1) and (2, 3), ...
    assert enss[0].tolist() == [0, 2, 1, 3]
    assert enss[1].tolist() == [1, 3, 0, 2]
    assert np.all(acc == 1.0)


def test_hrem_with_thermostats_keeps_the_segment_energy_in_its_column():
    """test2 runs its replicas with ORAC's thermostats: under them the energy
    record's column 15 still holds the REM segment energy (the thermostats'
    energy goes into the total only), so the exchange reads the same quantity
    -- a massive thermostat (1 cm^-1) leaves it at the NVE run's to 1e-7 after
    one step -- and a thermostatted HREM batch exchanges as the NVE one."""
    s = system()

    def make(factor, thermo):
        e = Engine(s.copy())
        e.set_rem(s.rematom, 0, factor)
        if thermo:
            e.set_thermostat(300.0, *thermo)
        e.md_setup(SCHED["dt_h"], SCHED["lrespa"], SCHED["mrespa"], SCHED["nupdte"], SCHED["rshk"])
        return e

    a, b = make(0.8, None), make(0.8, (1.0, 1.0, 1.0))
    ra = a.md_run(1, energy_every=1)
    rb = b.md_run(1, energy_every=1)
    et = b.md_thermostat()[4]
    assert rb[0, 15] != et
    np.testing.assert_allclose(rb[0, 15], ra[0, 15], rtol=1e-7)
    np.testing.assert_allclose(rb[0, 10], ra[0, 10] + et, rtol=1e-7)
    a.close()
    b.close()
    ladder = hrem.ladder_geometric(4, 0.7)
    engines = [make(f, (10.0, 10.0, 10.0)) for f in ladder]
    h = hrem.HremBatch(engines, ladder, KT_300, seed=5)
    for _ in range(3):
        p = h.interval(3)
        assert np.all(np.isfinite(p)) and sorted(h.ens.tolist()) == [0, 1, 2, 3]
    h.close()
    for e in engines:
        e.close()
