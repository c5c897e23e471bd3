"""Builds tests/golden/liquid_drift_oracle.npz: the FP64 oracle's energy
records of 1,000 outer r-RESPA steps (4 ps; 4/2/0.5 fs, shells 5.0/7.5/10.0 A,
SPME 48^3 order 4, lists every 6 steps, SETTLE/RATTLE-rigid waters, NVE) of
the liquid-density 3,000-water box from its seeded start, one record every
10 steps (the layout of orac_gpu_md_run).  The GPU's energy conservation is
compared against it (tests/test_gpu_md.py, bench.py).

    python tests/golden/make_drift.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "orac-porting_b200"), os.path.join(ROOT, "oracle")]
import oracle  # noqa: E402
from orac_b200 import systems  # noqa: E402

NSTEPS, EVERY = 1000, 10


def main():
    s = systems.config1_liquid()
    a, b = oracle.Oracle(s.copy()).cself()
    t0 = time.time()
    md = oracle.OracleMD(s.copy(), 4.0, 2, 4, 6, "l", econst=a + b)
    rec = md.run(NSTEPS, energy_every=EVERY)
    md.close()
    path = os.path.join(HERE, "liquid_drift_oracle.npz")
    np.savez_compressed(path, rec=rec, nsteps=NSTEPS, every=EVERY, dt_h=4.0)
    print(path, rec.shape, f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
