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
