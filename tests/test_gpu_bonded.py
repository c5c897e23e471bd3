"""GPU parity of the intramolecular path (mts_intra_n0: fpbond, fpbend,
fitors; mts_intra_n1: fptors, fnb14, fnbgrp) against the FP64 oracle.

FP64 on both sides (the GPU adds forces with FP64 atomics): forces relative
RMS <= 1e-10, energies relative <= 1e-10.
"""
import numpy as np
import pytest

import oracle
from orac_b200 import systems

pytestmark = pytest.mark.gpu

TOL = 1e-10


def chain_system():
    s = systems.polymer_in_water(nchain=240, nwat=900, box=32.0, nfft=(36, 36, 36), order=5, group_size=5,
                                 name="polymer_small")
    rng = np.random.default_rng(11)
    quads = np.array([(i + 1, i + 2, i + 3, i + 4) for i in range(0, 236, 3)], dtype=np.int32)
    k = len(quads)
    s.itors = quads
    s.itors_a = np.where(np.arange(k) % 2 == 0, 1.0, 2.0)
    s.itors_b = rng.uniform(0.5, 2.0, k) * 4184.0 / 1e7
    s.itors_c = np.where(np.arange(k) % 2 == 0, 1.0, 0.0)
    s.bend_ub_r0 = np.full(len(s.bends), 2.5)
    s.bend_ub_k = np.full(len(s.bends), 0.3 * s.bend_k[0])
    s.tors_n = np.array([[1.0, -2.0, 3.0, -3.0, 4.0, 6.0][i % 6] for i in range(len(s.tors))])
    r = s.cartesian()
    r[:, :240] += rng.normal(0.0, 0.05, (3, 240))
    sc = np.linalg.inv(s.co) @ r
    s.xp0, s.yp0, s.zp0 = sc[0], sc[1], sc[2]
    return s


def rel_rms(F, Fref):
    return float(np.sqrt(((F - Fref) ** 2).sum() / (Fref ** 2).sum()))


def test_intra_n0_parity():
    from orac_b200.engine import Engine

    s = chain_system()
    o = oracle.Oracle(s.copy())
    g = Engine(s.copy())
    Fr, er = o.intra_n0()
    Fg, eg = g.intra_n0()
    assert rel_rms(Fg, Fr) <= TOL
    ref = [er["bond"][0], er["bond"][1], er["bend"][0], er["bend"][1], er["itors"][0], er["itors"][1]]
    np.testing.assert_allclose(eg, ref, rtol=TOL, atol=1e-300)


def test_intra_n1_parity():
    from orac_b200.engine import Engine

    s = chain_system()
    o = oracle.Oracle(s.copy())
    g = Engine(s.copy())
    Ft, et = o.intra_torsions()
    F14, e14 = o.fnb14()
    Fgp, egp = o.fnbgrp()
    Fg, eg = g.intra_n1()
    assert rel_rms(Fg, Ft + F14 + Fgp) <= TOL
    np.testing.assert_allclose(eg[:2], et, rtol=TOL)
    np.testing.assert_allclose(eg[2:6], e14, rtol=TOL, atol=1e-300)
    np.testing.assert_allclose(eg[6:10], egp, rtol=TOL, atol=1e-300)
    assert len(s.ingrp) > 0 and len(s.int14) > 0
