"""The serving request loop (orac_b200.serve.Service) on the CPU, driven by
a simulated executor with a virtual clock: every request finishes, a
system's segments run in arrival order and never overlap, the memory
budget is never exceeded, idle systems are evicted least recently used
first (their state returned to the host), and a large system that does not
fit is not overtaken by later systems that are not resident."""
import dataclasses

import numpy as np
import pytest

from orac_b200 import serve


@dataclasses.dataclass
class FakeSystem:
    ntap: int
    co: np.ndarray = dataclasses.field(default_factory=lambda: np.eye(3) * 10.0)
    xp0: np.ndarray = None
    yp0: np.ndarray = None
    zp0: np.ndarray = None
    vx: np.ndarray = None
    vy: np.ndarray = None
    vz: np.ndarray = None


class FakeEngine:
    def __init__(self, s, nbytes):
        self.s = s
        self.nbytes = nbytes
        self.ctx = object()
        self.closed = False
        self.steps = 0

    def footprint(self):
        return self.nbytes

    def collect(self):
        return 0

    def md_state(self):
        n = self.s.ntap
        return np.full((3, n), float(self.steps)), np.zeros((3, n))

    def close(self):
        self.closed = True


class FakeServer:
    """Virtual-clock executor: at most max_active segments run at once, each
    takes nsteps * cost(engine) seconds whatever else runs."""

    def __init__(self, budget, max_active, cost):
        self.t = 0.0
        self.budget = budget
        self.max_active = max_active
        self.cost = cost
        self.reserved = 0
        self.peak = 0
        self.pending = []
        self.running = []
        self.next = 1
        self.log = []

    def now(self):
        return self.t

    def wait(self, dt):
        self.t += max(dt, 1e-4)

    def reserve(self, n):
        if self.reserved + n > self.budget:
            return False
        self.reserved += n
        self.peak = max(self.peak, self.reserved)
        return True

    def unreserve(self, n):
        assert 0 <= n <= self.reserved
        self.reserved -= n

    def submit(self, eng, nsteps, tag, t_arrival):
        assert not eng.closed
        tk = self.next
        self.next += 1
        self.pending.append([tk, tag, t_arrival, eng, nsteps])
        return tk

    def poll(self):
        while self.pending and len(self.running) < self.max_active:
            tk, tag, ta, eng, n = self.pending.pop(0)
            self.running.append((tk, tag, ta, self.t, self.t + n * self.cost(eng), eng, n))
        out = []
        for r in list(self.running):
            if r[4] <= self.t:
                self.running.remove(r)
                r[5].steps += r[6]
                self.log.append((r[5].s, r[3], r[4]))
                out.append(serve.Finished(r[0], r[1], r[2], r[3], r[4], 0))
        return out


def make_service(budget, max_active=4, sizes=(1000, 2000, 4000), nsteps=10):
    systems = {k: FakeSystem(n) for k, n in enumerate(sizes)}
    ex = FakeServer(budget, max_active, cost=lambda e: 1e-6 * e.s.ntap)
    svc = serve.Service(ex, systems, lambda s: FakeEngine(s, 1000 * s.ntap), nsteps=nsteps,
                        estimate=lambda s: 1200 * s.ntap)
    return svc, ex, systems


def check_per_system_order(ex, results):
    by = {}
    for s, t0, t1 in ex.log:
        by.setdefault(id(s), []).append((t0, t1))
    for iv in by.values():
        iv.sort()
        for (a0, a1), (b0, b1) in zip(iv, iv[1:]):
            assert b0 >= a1  # a system's segments never overlap


def test_every_request_finishes_in_order_per_system():
    svc, ex, systems = make_service(budget=10 ** 9)
    arr = serve.poisson_arrivals(rate=200.0, duration=0.5, nsystems=3, seed=1)
    res = svc.run(arr, timeout=100.0)
    assert len(res) == len(arr)
    assert all(r["status"] == 0 for r in res)
    assert all(r["t_arrival"] <= r["t_start"] <= r["t_end"] for r in res)
    check_per_system_order(ex, res)
    # a system's requests start in arrival order
    for sid in range(3):
        rs = sorted((r for r in res if r["sid"] == sid), key=lambda r: r["rid"])
        assert all(a["t_start"] <= b["t_start"] for a, b in zip(rs, rs[1:]))
    assert svc.builds == 3 and svc.evictions == 0


def test_budget_is_never_exceeded_and_idle_systems_are_evicted():
    # room for the two smaller systems only, or the largest alone
    svc, ex, systems = make_service(budget=1200 * 4000 + 10)
    arr = [(0.001 * k, k % 3) for k in range(12)]
    res = svc.run(arr, timeout=100.0)
    assert len(res) == 12
    assert ex.peak <= ex.budget
    assert svc.evictions > 0 and svc.builds > 3
    check_per_system_order(ex, res)
    # an evicted system's state went back to the host System
    assert any(s.xp0 is not None for s in systems.values())
    svc.close()
    assert ex.reserved == 0


def test_large_system_is_not_overtaken_by_later_non_resident_ones():
    sizes = (4000, 1000, 1000, 1000)
    svc, ex, systems = make_service(budget=1200 * 4000 + 10, sizes=sizes, max_active=8)
    # system 1 is resident and busy when the large system 0 arrives; later
    # requests for systems 2 and 3 (not resident) must wait behind it
    arr = [(0.0, 1), (0.0001, 0), (0.0002, 2), (0.0003, 3)]
    res = {r["rid"]: r for r in svc.run(arr, timeout=100.0)}
    assert res[1]["t_start"] <= res[2]["t_start"]
    assert res[1]["t_start"] <= res[3]["t_start"]
    assert ex.peak <= ex.budget


def test_segments_overlap_up_to_the_slot_limit():
    svc, ex, systems = make_service(budget=10 ** 9, sizes=(1000,) * 6, max_active=3)
    arr = [(0.0, k) for k in range(6)]
    res = svc.run(arr, timeout=100.0)
    starts = sorted(r["t_start"] for r in res)
    ends = sorted(r["t_end"] for r in res)
    # three run together, the next three start as those finish
    assert starts[2] < ends[0] <= starts[3]


def test_poisson_arrivals_are_seeded_and_have_the_rate():
    a = serve.poisson_arrivals(20.0, 200.0, 7, seed=11)
    b = serve.poisson_arrivals(20.0, 200.0, 7, seed=11)
    assert a == b
    assert abs(len(a) / 200.0 - 20.0) < 1.0
    assert {s for _, s in a} == set(range(7))


def test_fifo_one_at_a_time():
    lat, end = serve.fifo_one_at_a_time([(0.0, 0), (0.5, 1), (3.0, 0)], [1.0, 1.0, 1.0])
    assert np.allclose(lat, [1.0, 1.5, 1.0]) and end == pytest.approx(4.0)


class StateEngine(FakeEngine):
    """A stand-in engine whose state moves with the steps it has run."""

    def md_state(self):
        x = self.s.cartesian() + 0.01 * self.steps
        v = np.full((3, self.s.ntap), 0.001 * (1 + self.steps))
        return x, v


def test_evicted_and_closed_systems_are_checkpointed_as_orac_restarts(tmp_path):
    from orac_b200 import oracio, systems, units

    sy = {k: systems.two_waters(sep=(3.0 + k, 0.0, 0.0)) for k in range(3)}
    ex = FakeServer(budget=2500, max_active=4, cost=lambda e: 1e-3)
    svc = serve.Service(ex, sy, lambda s: StateEngine(s, 1000), nsteps=5, estimate=lambda s: 1000,
                        checkpoint_dir=str(tmp_path))
    res = svc.run([(0.0, 0), (0.0, 1), (0.0, 2), (0.01, 0), (0.02, 1)], timeout=100.0)
    assert len(res) == 5 and svc.evictions > 0
    states = {sid: r.engine.md_state() for sid, r in svc.resident.items()}
    svc.close()
    for sid, s in sy.items():
        r = oracio.read_rst(str(tmp_path / f"{sid}.rst"), s.ntap)
        assert r["nstep"] == svc.steps[sid] and r["nstep"] % 5 == 0 and r["nstep"] > 0
        assert np.allclose(r["co"], s.co) and np.allclose(r["oc"], np.linalg.inv(s.co))
        if sid in states:  # resident at close
            x, v = states[sid]
        else:  # evicted: its state went back to the host System too
            x = s.xyz_restart
            v = np.stack([s.vx, s.vy, s.vz])
        assert np.array_equal(r["xyz"], x) and np.array_equal(r["v"], v)
        ekin = 0.5 * float((np.asarray(s.mass) * (v * v).sum(0)).sum())
        ndf = 3 * s.ntap - len(np.asarray(s.constraints).reshape(-1, 2)) - 3
        assert r["temp"] == pytest.approx(units.kinetic_temperature(ekin, ndf), rel=1e-12)


def test_orac_restart_round_trip_rebuilds_the_system(tmp_path):
    """The real system's state written as an ORAC restart and read back
    rebuilds the same System with the fixture's topology (ORAC's own
    topology-parameter arrays)."""
    import os

    from orac_b200 import oracio, systems

    fix = np.load(os.path.join(os.path.dirname(__file__), "golden", "f0_fkbp12.npz"))
    tp, rst = oracio.split_arrays(dict(fix))
    sh = systems.Shells(rcutm=5.1, rtolm=0.3, rneim=0.4, rcutl=7.8, rtoll=0.3, rneil=0.5, rcuth=10.0, rtolh=0.3,
                        rneih=1.5)
    kw = dict(alphal=0.37, nfft=(48, 48, 48), order=4, shells=sh, ncell=(18, 18, 18))
    s = oracio.system_from_orac(tp, rst, **kw)
    path = str(tmp_path / "f0.rst")
    oracio.write_system_rst(path, s, rst["xyz"], rst["v"], nstep=30)
    r = oracio.read_rst(path, s.ntap)
    assert r["nstep"] == 30 and np.array_equal(r["xyz"], rst["xyz"]) and np.array_equal(r["v"], rst["v"])
    s2 = oracio.system_from_orac(tp, r, **kw)
    assert np.array_equal(s2.cartesian(), s.cartesian()) and np.array_equal(s2.vx, s.vx)


def test_prewarm_builds_what_the_budget_holds_and_requests_start_without_builds():
    """Service.prewarm builds the systems' contexts before requests arrive,
    within the budget and without evicting; requests for them then start
    without a build."""
    svc, ex, systems = make_service(budget=1200 * (1000 + 2000) + 10)
    assert svc.prewarm() == 2  # the largest system does not fit beside them
    assert svc.builds == 2 and svc.evictions == 0 and ex.reserved <= ex.budget
    res = svc.run([(0.0, 0), (0.001, 1), (0.002, 0)], timeout=100.0)
    assert len(res) == 3 and svc.builds == 2
    svc2, ex2, _ = make_service(budget=10 ** 9)
    assert svc2.prewarm() == 3 and svc2.prewarm() == 0  # built once
