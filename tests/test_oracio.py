"""ORAC file formats (orac_b200.oracio) on the CPU: the list-directed
record rules, the real-system fixture F0 built from ORAC's own
topology-parameter and restart files, and the restart writer read back."""
import importlib.util
import os

import numpy as np
import pytest

from orac_b200 import oracio, systems

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "f0_fkbp12.npz")


def load_make_f0():
    spec = importlib.util.spec_from_file_location("make_f0", os.path.join(HERE, "golden", "make_f0.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_list_directed_records(tmp_path):
    p = tmp_path / "r.txt"
    p.write_text("1 2 3 extra\n4 5\n\n6\n7 8\n9*2.5 0.5D0\n")
    r = oracio._Records(str(p))
    assert list(r.ints(2)) == [1, 2]  # the rest of the line is skipped
    assert list(r.ints(2)) == [4, 5]
    assert r.read(0) == []  # an empty READ consumes a record
    assert list(r.ints(3)) == [6, 7, 8]  # a READ spans records
    v = r.floats(10)
    assert np.allclose(v, [2.5] * 9 + [0.5])


def test_f0_fixture_builds_the_real_system():
    tp, rst = oracio.split_arrays(dict(np.load(FIX)))
    sh = systems.Shells(rcutm=5.1, rtolm=0.3, rneim=0.4, rcutl=7.8, rtoll=0.3, rneil=0.5, rcuth=10.0, rtolh=0.3,
                        rneih=1.5)
    s = oracio.system_from_orac(tp, rst, alphal=0.37, nfft=(48, 48, 48), order=4, shells=sh, ncell=(18, 18, 18))
    assert (s.ntap, s.ngrp, s.nprot, s.ntype) == (14900, 5082, 4397, 90)
    assert (s.ss_index == 1).sum() == 1715
    assert int((s.grppt[:, 1] - s.grppt[:, 0] + 1).max()) == 4
    assert abs(s.charge.sum()) < 1e-3 * np.abs(s.charge).sum() / len(s.charge)
    # the file's 5,732 proper and 339 improper torsions; ORAC's MD driver
    # moves 49 fast propers to the impropers (its topology table: 388)
    assert len(s.int14) == 4500 and len(s.tors) == 5732 - 49 and len(s.itors) == 388
    s0 = oracio.system_from_orac(tp, rst, alphal=0.37, nfft=(48, 48, 48), order=4, shells=sh, ncell=(18, 18, 18),
                                 move_fast_torsions=False)
    assert len(s0.tors) == 5732 and len(s0.itors) == 339
    # box from the restart: cubic, 54.616 A
    assert np.allclose(np.diag(s.co) * 2.0, 54.616, atol=1e-3)
    # the positions come back through the scaled frame
    assert np.allclose(s.cartesian(), rst["xyz"], atol=1e-12)


def test_fixture_matches_the_reference_files():
    """Regenerates the fixture from a reference checkout named by the
    ORAC_REFERENCE environment variable (skipped when it is not set)."""
    m = load_make_f0()
    root = os.environ.get("ORAC_REFERENCE", "")
    if not root or not os.path.isdir(os.path.join(root, "test1")):
        pytest.skip("no reference checkout (set ORAC_REFERENCE)")
    fresh = m.build_arrays(root)
    saved = dict(np.load(FIX))
    assert set(fresh) == set(saved)
    for k in fresh:
        assert np.array_equal(np.asarray(fresh[k]), saved[k]), k


def test_restart_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    co = np.diag([12.5, 13.0, 14.25])
    x = rng.uniform(-10, 10, (3, 50))
    v = rng.normal(0, 0.01, (3, 50))
    p = str(tmp_path / "s.rst")
    oracio.write_rst(p, co, x, v, nstep=7, temp=300.5, ngrp=4, nprot=2)
    r = oracio.read_rst(p, 50)
    assert np.array_equal(r["co"], co) and np.array_equal(r["xyz"], x) and np.array_equal(r["v"], v)
    assert r["nstep"] == 7 and r["temp"] == 300.5 and (r["ngrp"], r["nprot"]) == (4, 2)


def test_restart_round_trip_with_thermostats(tmp_path):
    """A thermostatted run's restart carries ORAC's hoover records (gh = eta,
    vh = etap, vh1), src/readrs.f:247-251; a restart without them reads as
    before."""
    rng = np.random.default_rng(4)
    co = np.diag([20.0, 20.0, 20.0])
    x = rng.uniform(-10, 10, (3, 12))
    v = rng.normal(0, 0.01, (3, 12))
    eta, etap = np.array([1e-3, -2e-4, 5e-3]), np.array([3e-5, -1e-6, 2e-4])
    p = str(tmp_path / "t.rst")
    oracio.write_rst(p, co, x, v, nstep=3, temp=298.0, thermostat=(eta, etap))
    r = oracio.read_rst(p, 12)
    assert np.array_equal(r["eta"], eta) and np.array_equal(r["etap"], etap)
    assert np.array_equal(r["xyz"], x) and np.array_equal(r["v"], v)
    q = str(tmp_path / "n.rst")
    oracio.write_rst(q, co, x, v)
    assert "eta" not in oracio.read_rst(q, 12)
