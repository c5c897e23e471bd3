"""Batched systems: one graph launch per H step advances every system, and
each system's trajectory is bitwise the one it follows alone (fixed-point
force sums make the result independent of what else runs on the device)."""
import numpy as np
import pytest

from orac_b200 import systems
from orac_b200.engine import Batch, Engine

pytestmark = pytest.mark.gpu


def replica(seed):
    s = systems.water_box(nwat=1000, box=31.1, lattice=10, seeds=(1, 2, 3, 40 + seed), nfft=(32, 32, 32),
                          name=f"water1000_r{seed}")
    return s


def test_batch_matches_alone_bitwise():
    nrep, nsteps = 4, 8
    alone = []
    for r in range(nrep):
        e = Engine(replica(r))
        e.md_setup(4.0, 2, 4, 6, "l")
        e.md_run(nsteps)
        alone.append(e.md_state())
        e.close()
    engines = []
    for r in range(nrep):
        e = Engine(replica(r))
        e.md_setup(4.0, 2, 4, 6, "l")
        engines.append(e)
    b = Batch(engines)
    b.run(nsteps)
    for r, e in enumerate(engines):
        x, v = e.md_state()
        assert np.array_equal(x, alone[r][0]), f"replica {r} positions differ"
        assert np.array_equal(v, alone[r][1]), f"replica {r} velocities differ"
    b.close()
    for e in engines:
        e.close()


def test_batched_energy_records_match_alone_bitwise():
    """Energy steps captured as graphs: a batch that writes each system's
    energy record every third step gives, per system, bitwise the state of
    that system run alone through md_run's energy steps (the host path) and
    the same records to 1e-11 (the FP64 energy sums are block sums added
    atomically, in no fixed order), and the records kept on the device
    equal the ones md_run returns (apart from the record number in
    column 0)."""
    nrep, nsteps, every = 3, 9, 3
    alone, alone_dev = [], []
    for r in range(nrep):
        e = Engine(replica(r))
        e.md_setup(4.0, 2, 4, 6, "l")
        rec = e.md_run(nsteps, energy_every=every)
        dev, n = e.md_records()
        assert n == nsteps // every
        np.testing.assert_array_equal(dev[:, 1:], rec[:, 1:])
        alone.append((rec, e.md_state()))
        e.close()
    engines = []
    for r in range(nrep):
        e = Engine(replica(r))
        e.md_setup(4.0, 2, 4, 6, "l")
        engines.append(e)
    b = Batch(engines)
    b.run(nsteps, energy_every=every)
    for r, e in enumerate(engines):
        dev, n = e.md_records()
        assert n == nsteps // every
        np.testing.assert_allclose(dev[:, 1:], alone[r][0][:, 1:], rtol=1e-11, atol=1e-11,
                                   err_msg=f"replica {r} records")
        x, v = e.md_state()
        assert np.array_equal(x, alone[r][1][0]) and np.array_equal(v, alone[r][1][1]), f"replica {r} state"
    b.close()
    for e in engines:
        e.close()


@pytest.mark.parametrize("tuning", [(16, 16, 5), (32, 16, 8), (16, 32, 6)])
def test_pair_launch_configuration_changes_speed_only(tuning):
    """The real-space kernel's lanes per group and occupancy (what the
    autotuner chooses) leave the trajectory bitwise unchanged: its i-atom
    sums are fixed point, independent of which lane took which pair."""
    ref = Engine(replica(0))
    ref.md_setup(4.0, 2, 4, 6, "l")
    ref.md_run(7)
    x0, v0 = ref.md_state()
    ref.close()
    e = Engine(replica(0))
    e.set_pair_tuning(*tuning)
    e.md_setup(4.0, 2, 4, 6, "l")
    e.md_run(7)
    assert e.pair_tuning() == tuning
    x, v = e.md_state()
    e.close()
    assert np.array_equal(x, x0) and np.array_equal(v, v0)


def test_batch_autotuner_persists_its_choice(tmp_path):
    cache = str(tmp_path / "pair_tuning.txt")
    engines = []
    for r in range(2):
        e = Engine(replica(r))
        e.md_setup(4.0, 2, 4, 6, "l")
        engines.append(e)
    b = Batch(engines)
    best, ms = b.tune(trial=2, cache=cache)
    assert best[0] in (16, 32) and best[1] in (16, 32) and best[2] in (5, 6, 8) and ms > 0.0
    assert all(e.pair_tuning() == best for e in engines)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and "batch;systems=2" in lines[0]
    again, ms2 = b.tune(trial=2, cache=cache)  # found in the cache: applied without timing
    assert again == best and ms2 == pytest.approx(ms, rel=1e-6)
    assert len(open(cache).read().splitlines()) == 1
    b.run(3)
    b.close()
    for e in engines:
        e.close()
