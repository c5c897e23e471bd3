"""Serving on the GPU: MD segments through the native executor
(orac_gpu_server_*) and the request loop (orac_b200.serve.Service).

- A segment's result is bitwise the same alone and in a mix of segments
  running concurrently on other streams (fixed-point force sums do not
  depend on what else runs), and the same as orac_gpu_md_run on its own.
- A built context's footprint is positive and below the estimate the
  request loop reserves before building it.
- With a memory budget that holds two of three systems the loop evicts
  idle systems (state back to the host) and rebuilds them later; the peak
  reservation stays within the budget, every segment ends with status 0,
  and each system's final state matches its uninterrupted run's to 1e-6 A
  (a restart from the saved Cartesian positions and velocities recomputes
  the forces with the energy kernels and re-projects the velocities: the
  same values to rounding).  Each evicted system's last state is also in
  its ORAC restart file in the checkpoint directory.
"""
import numpy as np
import pytest

from orac_b200 import oracio, serve, systems
from orac_b200.engine import Engine

pytestmark = pytest.mark.gpu

SCHED = (4.0, 2, 4, 6, "l")
SIZES = (3000, 5000, 4000)
REM = (0.6, 0.8, 0.4)


def system(k):
    return systems.solvated_chains(SIZES[k], 2000 + k, 0.07, name=f"serve{k}")


def engine(s, rem):
    e = Engine(s.copy())
    e.set_rem(s.rematom, 0, rem)
    e.md_setup(*SCHED)
    return e


def wait_all(srv, n, timeout=120.0):
    t0 = srv.now()
    out = []
    while len(out) < n:
        out += srv.poll()
        assert srv.now() - t0 < timeout, "segments did not finish"
        srv.wait(1e-3)
    return out


def test_segment_alone_and_in_the_mix_bitwise():
    nsteps = 12
    sy = [system(k) for k in range(3)]
    ref = engine(sy[1], REM[1])
    ref.md_run(nsteps)
    x_run, v_run = ref.md_state()
    ref.close()
    srv = serve.Server(budget_bytes=8e9, max_active=8, chunk=3)
    a = engine(sy[0], REM[0])
    srv.submit(a, nsteps, 0)
    f = wait_all(srv, 1)
    assert f[0].status == 0 and a.collect() == 0
    x_alone, v_alone = a.md_state()
    a.close()
    engines = [engine(s, r) for s, r in zip(sy, REM)]
    for k, e in enumerate(engines):
        srv.submit(e, nsteps, k)
    fin = wait_all(srv, 3)
    assert all(q.status == 0 for q in fin)
    assert all(q.t_arrival <= q.t_start <= q.t_end for q in fin)
    assert all(e.collect() == 0 for e in engines)
    x, v = engines[0].md_state()
    assert np.array_equal(x, x_alone) and np.array_equal(v, v_alone)
    x, v = engines[1].md_state()
    assert np.array_equal(x, x_run) and np.array_equal(v, v_run)
    st = srv.stats()
    assert st["steps_launched"] == 4 * nsteps and st["finished"] == 4
    srv.close()
    for e in engines:
        e.close()


def test_footprint_is_below_the_reserved_estimate():
    for k in range(3):
        s = system(k)
        e = engine(s, REM[k])
        fp = e.footprint()
        est = serve.estimate_footprint(s)
        e.close()
        assert 0 < fp <= est, (s.ntap, fp, est)


def test_service_evicts_within_budget_and_restarts_exactly(tmp_path):
    nsteps = 6
    sy = {k: system(k) for k in range(3)}
    base = {k: s.copy() for k, s in sy.items()}
    fp = {}
    for k, s in sy.items():
        e = engine(s, REM[k])
        fp[s.name] = e.footprint()
        e.close()
    est = sorted(fp.values())
    budget = est[1] + est[2] + 1  # two systems resident at most
    srv = serve.Server(budget_bytes=budget, max_active=4, chunk=2)
    svc = serve.Service(srv, sy, lambda s: engine(s, REM[int(s.name[-1])]), nsteps=nsteps,
                        estimate=lambda s: fp[s.name], checkpoint_dir=str(tmp_path))
    arr = [(0.0, 0), (0.0, 1), (0.0, 2), (0.05, 0), (0.05, 1), (0.05, 2)]
    res = svc.run(arr, timeout=300.0)
    assert len(res) == 6 and all(r["status"] == 0 for r in res)
    st = srv.stats()
    assert st["peak_reserved"] <= budget
    assert svc.evictions > 0
    # final states against uninterrupted runs of 2 segments each
    for k in range(3):
        if k in svc.resident:
            x, v = svc.resident[k].engine.md_state()
        else:
            x = sy[k].xyz_restart
        e = engine(base[k], REM[k])
        e.md_run(2 * nsteps)
        xr, _ = e.md_state()
        e.close()
        assert np.abs(x - xr).max() < 1e-6, (k, np.abs(x - xr).max())
        if k not in svc.resident:  # evicted: its last state is also an ORAC restart file
            r = oracio.read_rst(str(tmp_path / f"{k}.rst"), sy[k].ntap)
            assert np.array_equal(r["xyz"], x) and r["nstep"] == svc.steps[k]
    svc.close()
    srv.close()
