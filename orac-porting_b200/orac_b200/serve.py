"""Serving: MD segment requests for many systems on one GPU.

ORAC runs one system per process (src/mtsmd.f) and has no request loop;
this module is the host side of a service that keeps systems resident on
the device and runs segment requests as they arrive:

- `Server` wraps the native executor (orac_gpu_server_*, csrc/serve.cu):
  the device-memory budget, the segment slots and the pump thread that
  launches every running segment's step graphs on its own stream, so
  segments that arrive while others run overlap with them on the device.
- `Service` is the request loop: requests wait first come first served;
  a request for a resident, idle system starts at once; a request for a
  system that is not resident reserves its estimated footprint (evicting
  idle residents, least recently used first, when the budget is short:
  their state goes back to the host System), builds the system's context
  and starts.  A finished segment leaves its system resident.  With a
  checkpoint directory, every system whose state leaves the device (evicted,
  or resident at close) is also written as an ORAC restart file,
  `<system id>.rst`, which ORAC reads (src/readrs.f) and
  `oracio.load` / `oracio.read_rst` read back; systems can be submitted
  from ORAC's own files with `oracio.load`.

The loop is independent of the executor: the unit tests drive it with a
simulated executor on the CPU.
"""
from __future__ import annotations

import collections
import ctypes as C
import dataclasses
import math
import os
import time

import numpy as np

from . import lib as L


@dataclasses.dataclass
class Finished:
    ticket: int
    tag: int
    t_arrival: float
    t_start: float
    t_end: float
    status: int


class Server:
    """The native executor (orac_gpu_server_*)."""

    def __init__(self, device=0, budget_bytes=150e9, max_active=32, chunk=4):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.orac_gpu_server_create(device, int(budget_bytes), int(max_active), int(chunk), C.byref(h))
        if rc != L.ORAC_OK:
            raise L.OracGpuError(f"orac_gpu_server_create: {L.ERRORS.get(rc, rc)}")
        self.h = h
        self.budget = int(budget_bytes)

    def _check(self, rc, what):
        if rc != L.ORAC_OK:
            raise L.OracGpuError(f"{what}: {L.ERRORS.get(rc, rc)} {self.lib.orac_gpu_server_last_error(self.h).decode()}")

    def now(self):
        return self.lib.orac_gpu_server_now()

    def wait(self, seconds):
        time.sleep(seconds)

    def reserve(self, nbytes):
        g = C.c_int(0)
        self._check(self.lib.orac_gpu_server_reserve(self.h, int(nbytes), C.byref(g)), "server_reserve")
        return bool(g.value)

    def unreserve(self, nbytes):
        self._check(self.lib.orac_gpu_server_unreserve(self.h, int(nbytes)), "server_unreserve")

    def submit(self, engine, nsteps, tag, t_arrival=0.0):
        t = C.c_int64(0)
        self._check(self.lib.orac_gpu_server_submit(self.h, engine.ctx, int(nsteps), int(tag), float(t_arrival),
                                                    C.byref(t)), "server_submit")
        return t.value

    def poll(self, max_n=256):
        tk = np.zeros(max_n, np.int64)
        tg = np.zeros(max_n, np.int64)
        tm = np.zeros(3 * max_n)
        st = np.zeros(max_n, np.int32)
        n = C.c_int(0)
        self._check(self.lib.orac_gpu_server_poll(self.h, max_n, tk.ctypes.data, tg.ctypes.data, tm.ctypes.data,
                                                  st.ctypes.data, C.byref(n)), "server_poll")
        return [Finished(int(tk[k]), int(tg[k]), tm[3 * k], tm[3 * k + 1], tm[3 * k + 2], int(st[k]))
                for k in range(n.value)]

    def stats(self):
        a = (C.c_int64 * 8)()
        self._check(self.lib.orac_gpu_server_stats(self.h, a), "server_stats")
        keys = ("pending", "running", "finished_unpolled", "submitted", "finished", "reserved", "peak_reserved",
                "steps_launched")
        return dict(zip(keys, list(a)))

    def close(self):
        if self.h:
            self.lib.orac_gpu_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def estimate_footprint(s, lists=3, slack=1.25):
    """Device bytes a context of System `s` will hold, estimated before it
    is built (orac_gpu_footprint gives the exact figure after): the three
    nested neighbour lists (capacity 1.25 x the outer list's group pairs,
    12 bytes per entry), per-atom state and forces, the SPME grids, plus a
    fixed part.  Deliberately above the measured footprints of the
    solvated systems, so an admitted system seldom needs more than it
    reserved."""
    sh = s.shells
    rl = sh.rcuth + sh.rtolh + sh.rneih
    vol = abs(np.linalg.det(2.0 * np.asarray(s.co)))
    pairs = s.ngrp * (4.0 / 3.0 * math.pi * rl ** 3 * s.ngrp / vol) / 2.0
    n1, n2, n3 = s.nfft
    grid = n1 * n2 * n3
    return int(lists * slack * pairs * 12 + 1024 * s.ntap + 48 * grid + 64 * 2 ** 20)


@dataclasses.dataclass
class _Resident:
    engine: object
    nbytes: int
    busy: bool = False
    last: float = 0.0


@dataclasses.dataclass
class _Request:
    rid: int
    sid: int
    t_arrival: float


class Service:
    """Continuous-batching request loop.

    executor: a `Server` (or an object with its methods);
    systems: {system id: host System}; make_engine(system) -> an engine set
    up for MD (orac_b200.engine.Engine after md_setup, or a stand-in with
    .ctx, .footprint(), .collect(), .md_state(), .close());
    estimate(system) -> bytes to reserve before building;
    checkpoint_dir: where evicted and closed systems' states go as ORAC
    restart files (None: host memory only)."""

    def __init__(self, executor, systems, make_engine, nsteps=500, estimate=estimate_footprint, checkpoint_dir=None):
        self.ex = executor
        self.systems = systems
        self.make_engine = make_engine
        self.nsteps = nsteps
        self.estimate = estimate
        self.resident = {}
        self.waiting = collections.deque()
        self.tickets = {}
        self.results = []
        self.builds = 0
        self.evictions = 0
        self.checkpoint_dir = checkpoint_dir
        self.steps = collections.Counter()  # MD steps each system has run here

    # -------------------------------------------------------------- memory
    def _evict_one(self, protect):
        idle = [(r.last, sid) for sid, r in self.resident.items() if not r.busy and sid not in protect]
        if not idle:
            idle = [(r.last, sid) for sid, r in self.resident.items() if not r.busy]
        if not idle:
            return False
        _, sid = min(idle)
        r = self.resident.pop(sid)
        x, v = r.engine.md_state()
        self.checkpoint(sid, x, v)
        s = self.systems[sid]
        sc = np.linalg.inv(np.asarray(s.co)) @ x
        s.xp0, s.yp0, s.zp0 = sc[0].copy(), sc[1].copy(), sc[2].copy()
        s.xyz_restart = np.ascontiguousarray(x)
        s.vx, s.vy, s.vz = v[0].copy(), v[1].copy(), v[2].copy()
        r.engine.close()
        self.ex.unreserve(r.nbytes)
        self.evictions += 1
        return True

    def _reserve(self, nbytes, protect):
        while not self.ex.reserve(nbytes):
            if not self._evict_one(protect):
                return False
        return True

    def prewarm(self, sids=None):
        """Build the contexts of the given systems (all by default) before
        requests arrive, as far as the budget holds them without evicting,
        and capture their step graphs with one step each (a step the
        segments' counts leave out).  Returns the number built."""
        n = 0
        for sid in (self.systems if sids is None else sids):
            if sid in self.resident:
                continue
            s = self.systems[sid]
            need = int(self.estimate(s))
            if not self.ex.reserve(need):
                break
            eng = self.make_engine(s)
            self.builds += 1
            actual = int(eng.footprint())
            if actual > need and not self.ex.reserve(actual - need):
                eng.close()
                self.ex.unreserve(need)
                break
            if actual < need:
                self.ex.unreserve(need - actual)
            run = getattr(eng, "md_run", None)
            if run is not None:
                run(1)
            self.resident[sid] = _Resident(eng, actual)
            n += 1
        return n

    # ------------------------------------------------------------ requests
    def _start(self, req, r):
        r.busy = True
        t = self.ex.submit(r.engine, self.nsteps, req.rid, req.t_arrival)
        self.tickets[t] = req

    def _admit(self):
        memory_blocked = False
        protect = {q.sid for q in self.waiting}
        for req in list(self.waiting):
            r = self.resident.get(req.sid)
            if r is not None:
                if not r.busy and not any(q.sid == req.sid for q in self.waiting if q.rid < req.rid):
                    self.waiting.remove(req)
                    self._start(req, r)
                continue
            if memory_blocked or any(q.sid == req.sid for q in self.waiting if q.rid < req.rid):
                continue
            s = self.systems[req.sid]
            need = int(self.estimate(s))
            if not self._reserve(need, protect - {req.sid}):
                memory_blocked = True  # later non-resident systems wait behind this one
                continue
            eng = self.make_engine(s)
            self.builds += 1
            actual = int(eng.footprint())
            if actual > need and not self._reserve(actual - need, protect):
                eng.close()
                self.ex.unreserve(need)
                memory_blocked = True
                continue
            if actual < need:
                self.ex.unreserve(need - actual)
            r = _Resident(eng, actual)
            self.resident[req.sid] = r
            self.waiting.remove(req)
            self._start(req, r)

    def _finish(self, f):
        req = self.tickets.pop(f.ticket)
        r = self.resident[req.sid]
        r.busy = False
        r.last = f.t_end
        status = f.status
        if status == L.ORAC_OK:
            status = r.engine.collect()
        if status == L.ORAC_OK:
            self.steps[req.sid] += self.nsteps
        self.results.append(dict(rid=req.rid, sid=req.sid, natoms=int(self.systems[req.sid].ntap),
                                 t_arrival=f.t_arrival, t_start=f.t_start, t_end=f.t_end,
                                 latency=f.t_end - f.t_arrival, status=status))

    def run(self, arrivals, timeout=None, idle_wait=2e-4):
        """arrivals: [(seconds after the start, system id)] in time order.
        Returns one result dict per request (in completion order)."""
        t0 = self.ex.now()
        nreq = len(arrivals)
        i = 0
        while len(self.results) < nreq:
            now = self.ex.now()
            if timeout is not None and now - t0 > timeout:
                raise TimeoutError(f"{len(self.results)} of {nreq} requests finished in {timeout} s")
            while i < nreq and t0 + arrivals[i][0] <= now:
                self.waiting.append(_Request(i, arrivals[i][1], t0 + arrivals[i][0]))
                i += 1
            if self.waiting:
                self._admit()
            done = self.ex.poll()
            for f in done:
                self._finish(f)
            if not done:
                nxt = (t0 + arrivals[i][0] - now) if i < nreq else idle_wait
                self.ex.wait(max(0.0, min(idle_wait, nxt)))
        return self.results

    def checkpoint(self, sid, x, v):
        """Write system `sid` at Cartesian positions x and velocities v as an
        ORAC restart file in the checkpoint directory (if one is set)."""
        if self.checkpoint_dir is None:
            return None
        from . import oracio

        os.makedirs(self.checkpoint_dir, exist_ok=True)
        path = os.path.join(self.checkpoint_dir, f"{sid}.rst")
        oracio.write_system_rst(path, self.systems[sid], x, v, nstep=self.steps[sid])
        return path

    def close(self):
        for sid, r in self.resident.items():
            if self.checkpoint_dir is not None:
                self.checkpoint(sid, *r.engine.md_state())
            r.engine.close()
            self.ex.unreserve(r.nbytes)
        self.resident.clear()


def poisson_arrivals(rate, duration, nsystems, seed):
    """Arrival times of a Poisson process of `rate` per second over
    `duration` seconds, each for a system drawn uniformly (seeded)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            return out
        out.append((t, int(rng.integers(nsystems))))


def fifo_one_at_a_time(arrivals, service_s):
    """Latencies of the same requests served one at a time, first come
    first served, when request k takes service_s[k] seconds on the device
    (the plain single-system path: one system at a time)."""
    free, lat = 0.0, []
    for (t, _), d in zip(arrivals, service_s):
        start = max(t, free)
        free = start + d
        lat.append(free - t)
    return np.array(lat), free
