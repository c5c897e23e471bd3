#!/usr/bin/env python
"""MD throughput (ns/day) of the B200 r-RESPA nonbonded force path.

One step = one outer r-RESPA step (H = 4 fs: 1 H shell, 2 L shells + SPME,
8 M shells, drift + SHAKE/RATTLE) of 3,000 rigid waters (9,000 atoms) at
liquid density (44.7 A box, alpha 0.35, SPME 48^3 order 4, shells
5.0/7.5/10.0 A, list update every 6 steps; `--workload config1` selects the
31 A box as specified, three times liquid density), run by the
device-resident driver of liborac_gpu.so with the state resident in HBM.
Further legs on the same line: the state's forces and energies against the
FP64 oracle, a per-kernel-family breakdown of the step, a 1,000-step energy
drift against the oracle's, 64 batched alchemical windows, ORAC's own test1
system (NVE, and with test1's Nose-Hoover thermostats), the 22,700-atom
solvated chain and the as-specified 31 A box,
replica exchange of 16 batched replicas, test4's non-equilibrium work swarm
on ORAC's system, 128 uneven HREM replicas and the serving loop.  Prints
one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU restatement of ORAC's loop (the oracle, FP64,
OpenMP over all host cores) on the same workload.  Under torchrun each rank
runs an independent replica (the path does not shard within one system).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# batched systems are parallel graph branches: let the device run 32 at a time
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
for p in (os.path.join(ROOT, "orac-porting_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

from orac_b200 import systems, units  # noqa: E402

FS_PER_DAY = 86400.0e15  # fs per day of wall time per 1 fs/s
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 74.4: used only if the FMA-rate probe fails
METRIC = "MD ns/day and p50/p99 segment latency, batched vs plain, at force err<=1e-5"

WORKLOADS = {
    "config1": dict(build=systems.config1_water, dt_h=4.0, lrespa=2, mrespa=4, nupdte=6, rshk="l",
                    desc="3,000 rigid 3-site waters (9,000 atoms), 31.0 A cubic box, alpha 0.35, SPME 32^3 "
                         "order 4, r-RESPA 0.5/2/4 fs with shells 5.0/7.5/10.0 A, list update every 6 H steps"),
    "liquid": dict(build=systems.config1_liquid, dt_h=4.0, lrespa=2, mrespa=4, nupdte=6, rshk="l",
                   desc="3,000 rigid 3-site waters (9,000 atoms) of the 31 A workload at liquid density: 44.7 A "
                        "cubic box, alpha 0.35, SPME 48^3 order 4, r-RESPA 0.5/2/4 fs with shells 5.0/7.5/10.0 A, "
                        "list update every 6 H steps"),
}


def f0_system():
    """The reference's test1 system as ORAC assembled it (fixture F0:
    solvated FKBP12 with its ligand, 14,900 atoms, from ORAC's own
    topology-parameter and restart files), with test1's parameters: SPME
    alpha 0.37 on 48^3 order 4, shells 5.1/7.8/10.0 A, 18^3 linked cells,
    bonds to hydrogen rigid (STRETCHING HEAVY)."""
    from orac_b200 import oracio

    tp, rst = oracio.split_arrays(dict(np.load(os.path.join(ROOT, "tests", "golden", "f0_fkbp12.npz"))))
    sh = systems.Shells(rcutm=5.1, rtolm=0.3, rneim=0.4, rcutl=7.8, rtoll=0.3, rneil=0.5, rcuth=10.0, rtolh=0.3,
                        rneih=1.5)
    return oracio.system_from_orac(tp, rst, alphal=0.37, nfft=(48, 48, 48), order=4, shells=sh, ncell=(18, 18, 18),
                                   fudge=0.83333, lj_fudge=0.5, name="F0_fkbp12", rigid_hydrogen=True)


def f0_test4_system(k):
    """F0 at test2's restart state k (0 ij4i0000, 1 ij4i0001, 2 ij4i0003)
    with the reference's test4 parameters: shells 5.0/8.1/12.5 A, SPME alpha
    0.37 on 48 x 49 x 48 order 4, bonds to hydrogen rigid, the ligand (atoms
    1-52) the removed alchemical species."""
    from orac_b200 import oracio

    gold = os.path.join(ROOT, "tests", "golden")
    tp, rst = oracio.split_arrays(dict(np.load(os.path.join(gold, "f0_fkbp12.npz"))))
    if k > 0:
        r = np.load(os.path.join(gold, "f0_orac_records.npz"))
        rst = dict(rst, co=r[f"co{k}"], xyz=r[f"xyz{k}"], v=r[f"v{k}"])
    sh = systems.Shells(rcutm=5.0, rtolm=0.3, rneim=0.5, rcutl=8.1, rtoll=0.3, rneil=0.5, rcuth=12.5, rtolh=0.3,
                        rneih=1.5)
    s = oracio.system_from_orac(tp, rst, alphal=0.37, nfft=(48, 49, 48), order=4, shells=sh, ncell=(18, 18, 18),
                                fudge=0.83333, lj_fudge=0.5, name=f"F0_test4_{k}", rigid_hydrogen=True)
    ss = np.ones(s.ntap, np.int32)
    ss[:52] = -2
    s.ss_alchemy = ss
    return s


# test4's NE run: 15/3/1.5/0.75/0.375 fs, lists every 60 fs, the shifted
# potential SHIFT-POT 4.0 0.35, the 1.5 ps schedule of 15.off
NE_WORKLOAD = dict(dt_h=15.0, lrespa=5, mrespa=2, n1respa=2, n0respa=2, nupdte=4, rshk="l")
NE_WALKERS = 12  # the three restart states, four velocity draws each

# the reference's test1 schedule: 15 fs outer step, L 3 fs (SPME), M 1.5 fs,
# intramolecular 0.75 / 0.375 fs, list update every 6 steps
F0_WORKLOAD = dict(build=f0_system, dt_h=15.0, lrespa=5, mrespa=2, n1respa=2, n0respa=2, nupdte=6, rshk="l")
# test1/md.in and test2/rem.in: TEMPERATURE 298, THERMOS solute/solvent/cofm 10 cm^-1
TEST1_THERMOS = (298.0, 10.0, 10.0, 10.0)
NVT_LIQUID = (300.0, 20.0, 20.0, 20.0)  # test3/test4's THERMOS (300 K, 20 cm^-1)
DUDL_STEPS, DUDL_EVERY = 400, 2  # dU/dlambda sampling of the batched windows
SERVE_PLAIN_SAMPLE = 8  # serving requests also run one at a time, to check the plain model
HREM_N, HREM_EVERY, HREM_INTERVALS = 16, 15, 10  # replica-exchange leg
# the pair-kernel autotuner's choices per device and workload shape
TUNE_CACHE = os.path.join(ROOT, "orac-porting_b200", "orac_b200", "pair_tuning.txt")
TUNE_TRIAL = 6


def tuned(obj):
    """Autotune a context or a batch (cached choices are applied without
    timing): the chosen configuration, its time per step, and whether it was
    measured in this run or read from the cache."""
    n0 = len(open(TUNE_CACHE).read().splitlines()) if os.path.exists(TUNE_CACHE) else 0
    best, ms = obj.tune(trial=TUNE_TRIAL, cache=TUNE_CACHE)
    n1 = len(open(TUNE_CACHE).read().splitlines()) if os.path.exists(TUNE_CACHE) else 0
    return {"lpg_m": best[0], "lpg_lh": best[1], "blocks_per_sm": best[2], "ms_per_step": ms,
            "source": "measured in this run" if n1 > n0 else "cache (orac_b200/pair_tuning.txt)"}
TEST1_PUBLISHED_NS_DAY = 4.41  # test1/md.out:1061,1063: 58.799 s for 3,000 fs, 8 OpenMP threads, NPT


def ns_per_day(steps, dt_h_fs, seconds):
    return steps * dt_h_fs * 1e-6 * 86400.0 / seconds


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def econst_of(s, engine=None):
    """Self energy (cself): the constant of the energy records (the erf
    corrections of the constraints are part of the records themselves)."""
    if engine is not None:
        a, b = engine.cself()
    else:
        import oracle

        a, b = oracle.Oracle(s).cself()
    return a + b


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(index), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for k, nm in enumerate(names):
                    if r[4 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def force_check(s, x):
    """Forces and energies of the Cartesian state x (3, N) through the C ABI
    (the three shells and SPME, lists built at x) against the FP64 oracle on
    the same positions: ORAC's check_force metric (relative RMS of the total
    force, src/pme_code.f:378-396) and the relative error of each energy
    term (LJ, real-space Coulomb, reciprocal) and of their sum."""
    import oracle
    from orac_b200.engine import Engine

    t = s.copy()
    sc = np.linalg.inv(np.asarray(s.co)) @ np.asarray(x)
    t.xp0, t.yp0, t.zp0 = sc[0].copy(), sc[1].copy(), sc[2].copy()
    g, o = Engine(t.copy()), oracle.Oracle(t.copy())
    try:
        g.update_lists()
        o.update_lists()
        Fg, Fo = np.zeros((3, s.ntap)), np.zeros((3, s.ntap))
        eg, eo = np.zeros(6), np.zeros(6)
        for sh in "mlh":
            F, en, _ = g.shell(sh)
            Fg += F
            eg += g.ue6(en)
            F, ue, _ = o.shell(sh)
            Fo += F
            eo += np.asarray(ue)
        F, rg, _ = g.fft_pme()
        Fg += F
        F, ro, _ = o.fft_pme()
        Fo += F
    finally:
        g.close()
    terms_g = {"lj": eg[:3].sum(), "coul_real": eg[3:].sum(), "reciprocal": rg}
    terms_o = {"lj": eo[:3].sum(), "coul_real": eo[3:].sum(), "reciprocal": ro}
    terms_g["total"] = sum(terms_g.values())
    terms_o["total"] = sum(terms_o.values())
    rel = {k: abs(terms_g[k] - terms_o[k]) / abs(terms_o[k]) for k in terms_o}
    return {"force_rel_rms": float(np.sqrt(((Fg - Fo) ** 2).sum() / (Fo ** 2).sum())),
            "energy_rel_err": max(rel.values()), "energy_rel_err_terms": rel,
            "energy_kjmol": {k: v * units.KJMOL for k, v in terms_o.items()},
            "how": "state after the timed steps: M, L, H shells and SPME through the C ABI (lists rebuilt at that "
                   "state) against the FP64 oracle on the same positions; force = sum of the four"}


def drift_fit(rec, dt_h):
    """Total-energy drift (kJ/mol per ps, least squares) and the RMS of the
    residual, of energy records."""
    t = rec[:, 0] * dt_h * 1e-3
    e = rec[:, 10] * units.KJMOL
    p = np.polyfit(t, e, 1)
    return float(p[0]), float(np.std(e - np.polyval(p, t)))


def drift_run(wl, s, device):
    """1,000 outer steps of the workload from its seeded start (NVE, energy
    record every 10 steps) on the device beside the FP64 oracle's run of the
    same 1,000 steps (tests/golden/liquid_drift_oracle.npz)."""
    from orac_b200.engine import Engine

    ref = np.load(os.path.join(ROOT, "tests", "golden", "liquid_drift_oracle.npz"))
    g = Engine(s.copy(), device=device)
    g.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], econst=econst_of(s, g))
    rec = g.md_run(int(ref["nsteps"]), energy_every=int(ref["every"]))
    g.close()
    dg, fg = drift_fit(rec, wl["dt_h"])
    do, fo = drift_fit(ref["rec"], float(ref["dt_h"]))
    return {"steps": int(ref["nsteps"]), "gpu_drift_kjmol_per_ps": dg, "gpu_rms_kjmol": fg,
            "oracle_drift_kjmol_per_ps": do, "oracle_rms_kjmol": fo,
            "total_energy_kjmol": float(rec[0, 10] * units.KJMOL),
            "how": "least-squares slope of the total energy and RMS of its residual over 1,000 outer steps (4 ps) "
                   "from the seeded start, records every 10 steps; oracle: the FP64 CPU restatement's run of the "
                   "same steps (fixture made by tests/golden/make_drift.py)"}


def fp32_peak(device):
    """Measured FP32 FMA rate of the device (orac_gpu_fp32_rate), TFLOP/s."""
    import ctypes as C

    from orac_b200 import lib

    L = lib.load()
    tf, ms = C.c_double(), C.c_double()
    if L.orac_gpu_fp32_rate(device, C.byref(tf), C.byref(ms)) != 0 or tf.value <= 0.0:
        return None
    return tf.value


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def ncu_traffic():
    """DRAM bytes per launch of the real-space kernel from the committed ncu
    summary (profiles/k_pair_liquid.json), or None."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "k_pair_liquid.json")))
        return float(d["dram_bytes_per_launch"])
    except Exception:
        return None


# ----------------------------------------------------------------------- CPU


def cpu_run(wl, s, steps, warmup, budget_s=None):
    """Oracle r-RESPA loop on all host cores; returns (seconds, steps, cores)."""
    import oracle

    cores = os.cpu_count() or 1
    md = oracle.OracleMD(s, wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], nthreads=cores,
                         n1respa=wl.get("n1respa", 1), n0respa=wl.get("n0respa", 1),
                         econst=0.0)
    if warmup:
        md.run(warmup)
    done, t = 0, 0.0
    while done < steps:
        t0 = time.perf_counter()
        md.run(1)
        t += time.perf_counter() - t0
        done += 1
        if budget_s is not None and t >= budget_s and done >= 3:
            break
    md.close()
    return t, done, cores


# ----------------------------------------------------------------------- GPU


def gpu_arm(args, wl, s, device):
    import ctypes as C

    import torch

    from orac_b200.engine import Engine

    torch.cuda.set_device(device)
    eng = Engine(s.copy(), device=device)
    L = eng.lib
    ec = econst_of(s, eng)
    eng.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], econst=ec)
    ws, rank, local = dist_info()
    # clocks sampled from the autotuner's and warm-up steps through the timed
    # steps: the timed region alone is shorter than nvidia-smi's 200 ms period
    clocks = ClockSampler(device) if rank == 0 else None
    tuning = tuned(eng)
    L.orac_gpu_prof_enable(eng.ctx, 1)
    stream = torch.cuda.ExternalStream(L.orac_gpu_get_stream(eng.ctx), device=device)
    def ok(rc, what):
        if rc:
            raise RuntimeError(f"{what}: status {rc}: {L.orac_gpu_last_error(eng.ctx).decode()}")

    # warm-up (also captures the step graphs)
    for _ in range(args.warmup):
        ok(L.orac_gpu_md_run_async(eng.ctx, 1), "md_run_async")
        ok(L.orac_gpu_md_collect(eng.ctx), "md_collect")
    cnt = (C.c_int64 * 4)()
    L.orac_gpu_counters(eng.ctx, cnt, 1)
    L.orac_gpu_prof_read(eng.ctx, None, None, 1)
    l0 = C.c_int64()
    L.orac_gpu_stats(eng.ctx, None, C.byref(l0))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")  # > 126 MB L2
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()  # L2 flushed between timed steps
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = L.orac_gpu_md_run_async(eng.ctx, 1)
        e1.record(stream)
        rc |= L.orac_gpu_md_collect(eng.ctx)
        if rc:
            raise RuntimeError(L.orac_gpu_last_error(eng.ctx).decode())
        ms = e0.elapsed_time(e1)
        step_ms.append(ms)
        total_ms += ms
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([total_ms], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    clk = clocks.stop() if clocks else None
    if clk:
        clk["window"] = "autotuner and warm-up steps through the timed steps"
    l1 = C.c_int64()
    L.orac_gpu_stats(eng.ctx, None, C.byref(l1))
    L.orac_gpu_counters(eng.ctx, cnt, 0)
    pms = C.c_double()
    pn = C.c_int64()
    L.orac_gpu_prof_read(eng.ctx, C.byref(pms), C.byref(pn), 0)
    res = dict(tuning=tuning, total_ms=total_ms, step_ms=step_ms, launches=int(l1.value - l0.value), scanned=cnt[0],
               kept=cnt[1],
               pairs_ewald=cnt[2], pairs_lj=cnt[3], kpair_ms=pms.value, kpair_n=int(pn.value), clocks=clk,
               kpair_how="CUDA events recorded as graph nodes around every k_pair launch of the timed steps")
    if res["kpair_n"] <= 0:
        # events inside the replayed graphs could not be timed: time the same
        # steps with direct launches (events bracket each k_pair launch)
        L.orac_gpu_md_set_graphs(eng.ctx, 0)
        L.orac_gpu_prof_read(eng.ctx, None, None, 1)
        nprof = min(args.steps, 10)
        for _ in range(nprof):
            flush.zero_()
            torch.cuda.synchronize()
            ok(L.orac_gpu_md_run_async(eng.ctx, 1), "md_run_async")
            ok(L.orac_gpu_md_collect(eng.ctx), "md_collect")
        L.orac_gpu_prof_read(eng.ctx, C.byref(pms), C.byref(pn), 0)
        L.orac_gpu_md_set_graphs(eng.ctx, 1)
        per_step = pn.value / nprof
        res["kpair_n"] = int(round(per_step * args.steps))
        res["kpair_ms"] = pms.value / max(1, pn.value) * res["kpair_n"]
        res["kpair_how"] = (f"CUDA events around each k_pair launch of {nprof} further steps launched directly "
                            "(graph-node events could not be timed)")
    # end-to-end through the public ABI with host buffers: every step copies
    # the state in from pinned host memory and reads it back
    n = s.ntap
    # one pinned buffer: x, y, z, vx, vy, vz back to back (two copies each way)
    hbuf = torch.empty(6 * n, dtype=torch.float64).pin_memory()
    host = [hbuf[k * n:(k + 1) * n] for k in range(6)]
    x, v = eng.md_state()
    for k in range(3):
        host[k].copy_(torch.from_numpy(x[k]))
        host[3 + k].copy_(torch.from_numpy(v[k]))
    ptrs = [h.data_ptr() for h in host]
    views = [h.numpy() for h in host]
    e2e_steps = max(3, min(args.steps, 20))
    t_e2e = 0.0
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = L.orac_gpu_md_set_state(eng.ctx, *ptrs)
        rc |= L.orac_gpu_md_run_async(eng.ctx, 1)
        rc |= L.orac_gpu_md_get_state(eng.ctx, *views)
        rc |= L.orac_gpu_md_collect(eng.ctx)
        t_e2e += time.perf_counter() - t0
        if rc:
            raise RuntimeError(L.orac_gpu_last_error(eng.ctx).decode())
    res["e2e_s"] = t_e2e
    res["e2e_steps"] = e2e_steps
    res["bytes_io"] = 6 * n * 8
    res["G"], res["N"] = s.ngrp, s.ntap
    res["shell_evals"] = args.steps * (1 + wl["lrespa"] + wl["lrespa"] * wl["mrespa"])
    try:
        res["step_breakdown"] = step_breakdown(eng, flush, max(5, min(args.steps, 20)))
    except Exception as exc:
        res["step_breakdown"] = {"error": f"{type(exc).__name__}: {exc}"}
    xs, _ = eng.md_state()
    eng.close()
    try:
        res["nvt"] = nvt_arm(args, wl, s, device, flush)
    except Exception as exc:
        res["nvt"] = {"error": f"{type(exc).__name__}: {exc}"}
    try:
        res["force_check"] = force_check(s, xs)
    except Exception as exc:
        res["force_check"] = {"error": f"{type(exc).__name__}: {exc}"}
    res["fp32_peak"] = fp32_peak(device)
    if args.drift and args.workload == "liquid":
        try:
            res["energy_conservation"] = drift_run(wl, s, device)
        except Exception as exc:
            res["energy_conservation"] = {"error": f"{type(exc).__name__}: {exc}"}
    if args.batch > 1:
        try:
            res["batched"] = batch_arm(args, wl, s, device, flush)
        except Exception as exc:  # reported in the JSON line; the plain leg stands on its own
            res["batched_error"] = f"{type(exc).__name__}: {exc}"
    if ws == 1 and args.f0:
        try:
            res["orac_test1"] = f0_arm(args, device, flush)
        except Exception as exc:
            res["orac_test1"] = {"error": f"{type(exc).__name__}: {exc}"}
    if ws == 1 and args.hrem:
        try:
            res["hrem"] = hrem_arm(args, wl, device)
        except Exception as exc:
            res["hrem"] = {"error": f"{type(exc).__name__}: {exc}"}
    if ws == 1 and args.ne:
        try:
            res["ne_swarm"] = ne_arm(args, device)
        except Exception as exc:
            res["ne_swarm"] = {"error": f"{type(exc).__name__}: {exc}"}
    if ws == 1 and args.configs:
        for key, arm in (("config2", config2_arm), ("config1_as_specified", config1_fixed_arm)):
            try:
                res[key] = arm(args, device, flush)
            except Exception as exc:
                res[key] = {"error": f"{type(exc).__name__}: {exc}"}
    if ws == 1 and args.uneven > 1:
        try:
            res["uneven"] = uneven_arm(args, wl, device, flush)
        except Exception as exc:
            res["uneven"] = {"error": f"{type(exc).__name__}: {exc}"}
    if ws == 1 and args.serve > 0:
        try:
            res["served"] = serve_arm(args, wl, device)
        except Exception as exc:
            res["served"] = {"error": f"{type(exc).__name__}: {exc}"}
    return res


PROF_FAMILIES = ("pair", "drift_kick", "spme", "bonded")


def step_breakdown(eng, flush, nsteps):
    """Device time per step of each kernel family, from CUDA events that
    bracket every launch of the family inside the captured step graphs (the
    pair kernel, the drift and kick kernels, one SPME evaluation from spread
    to gather, the bonded kernel), over nsteps further steps after the timed
    ones, L2 flushed before each.  The SPME evaluations run on the step's
    second stream, beside the pair kernels: the families' times can add up
    to more than the step."""
    import ctypes as C

    import torch

    L = eng.lib
    L.orac_gpu_prof_enable(eng.ctx, (1 << len(PROF_FAMILIES)) - 1)
    stream = torch.cuda.ExternalStream(L.orac_gpu_get_stream(eng.ctx), device=flush.device)
    for _ in range(2):  # captures the instrumented graphs
        L.orac_gpu_md_run_async(eng.ctx, 1)
        L.orac_gpu_md_collect(eng.ctx)
    L.orac_gpu_prof_read(eng.ctx, None, None, 1)
    status = []

    def one():
        # the events of a replayed step graph are read when the step is collected
        L.orac_gpu_md_run_async(eng.ctx, 1)
        status.append(L.orac_gpu_md_collect(eng.ctx))

    step_ms = _timed_steps(one, stream, flush, nsteps)
    if any(status):
        raise RuntimeError(L.orac_gpu_last_error(eng.ctx).decode())
    out = {"steps": nsteps, "ms_per_step": sum(step_ms) / nsteps,
           "how": "CUDA events recorded as graph nodes around each launch of the family (the event nodes break the "
                  "launches' programmatic overlap, so this step is a little slower than the timed one)"}
    for f, name in enumerate(PROF_FAMILIES):
        ms = C.c_double()
        n = C.c_int64()
        L.orac_gpu_prof_read_family(eng.ctx, f, C.byref(ms), C.byref(n), 0)
        if n.value < 0:
            out[name] = {"error": "some event pairs could not be timed"}
            continue
        out[name] = {"ms_per_step": ms.value / nsteps, "launches_per_step": n.value / nsteps,
                     "us_per_launch": 1e3 * ms.value / n.value if n.value else None,
                     "share_of_step": ms.value / sum(step_ms) if step_ms else None}
    L.orac_gpu_prof_enable(eng.ctx, 0)
    return out


def nvt_arm(args, wl, s, device, flush):
    """The plain workload with Nose-Hoover thermostats (ORAC's THERMOS at
    300 K, 20 cm^-1 each, as test3/test4 couple them): the same steps timed
    the same way, and the thermostats' state at the end."""
    import torch

    from orac_b200.engine import Engine

    e = Engine(s.copy(), device=device)
    e.set_thermostat(*NVT_LIQUID)
    e.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], econst=0.0)
    L = e.lib
    st = torch.cuda.ExternalStream(L.orac_gpu_get_stream(e.ctx), device=device)
    for _ in range(args.warmup):
        L.orac_gpu_md_run_async(e.ctx, 1)
    if e.collect():
        raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
    ms = _timed_steps(lambda: L.orac_gpu_md_run_async(e.ctx, 1), st, flush, args.steps)
    if e.collect():
        raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
    eta, etap, q, ndf, et = e.md_thermostat()
    e.close()
    return {"value": ns_per_day(args.steps, wl["dt_h"], sum(ms) / 1e3), "unit": "ns/day",
            "ms_per_step": sum(ms) / args.steps,
            "thermostats": f"Nose-Hoover (ORAC's THERMOS) at {NVT_LIQUID[0]:g} K, centres of mass, solute and "
                           f"solvent at {NVT_LIQUID[1]:g} cm^-1",
            "etap": [float(x) for x in etap], "ndf": [int(x) for x in ndf]}


def _timed_steps(run_one, stream, flush, steps):
    """CUDA-event time of each of `steps` calls of run_one on `stream`, L2
    flushed before each."""
    import torch

    out = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_one()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def window_lambdas(lam):
    """The two-stage removal path of ORAC's NE runs (test3/test4's schedule
    switches the charges off first, then the LJ): control lambda in [0, 0.5]
    takes lrmq from 0 to 1 with lrm = 0, lambda in [0.5, 1] takes lrm from
    0 to 1 with the charges off.  (ladd, lrm, laddq, lrmq) and their
    derivatives with respect to lambda."""
    if lam <= 0.5:
        return (0.0, 0.0, 0.0, 2.0 * lam), [0.0, 0.0, 0.0, 2.0]
    return (0.0, 2.0 * lam - 1.0, 0.0, 1.0), [0.0, 2.0, 0.0, 0.0]


def window_engine(base, k, nwin, device, wl):
    """Lambda window k at lambda = k / (nwin - 1) on the two-stage removal
    path (window_lambdas; soft core 0.5 0.5), dU/dlambda of that control
    lambda."""
    from orac_b200.engine import Engine

    lam = k / (nwin - 1)
    e = Engine(base.copy(), device=device)
    e.set_alchemy(base.ss_alchemy, 0.5, 0.5)
    lv, dl = window_lambdas(lam)
    e.set_lambda(*lv, dlam=dl)
    e.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], econst=0.0)
    return e, lam


def batch_arm(args, wl, s, device, flush):
    """The alchemical lambda-window batch: `args.batch` windows of the
    40-atom ligand in the liquid water box (lambda_k = k / (B - 1) on the
    two-stage removal path: charges, then LJ) advanced by one graph launch per outer step
    (orac_gpu_batch_run); the plain reference is one window alone on the
    same driver.  Every window ends with an energy step that yields its
    dU/dlambda."""
    import ctypes as C

    import torch

    from orac_b200.engine import Batch

    base = systems.ligand_in_water()
    nwin = args.batch
    # one window alone (plain)
    e1, _ = window_engine(base, nwin // 2, nwin, device, wl)
    tune_plain = tuned(e1)
    L = e1.lib
    st1 = torch.cuda.ExternalStream(L.orac_gpu_get_stream(e1.ctx), device=device)
    for _ in range(args.warmup):
        L.orac_gpu_md_run_async(e1.ctx, 1)
        L.orac_gpu_md_collect(e1.ctx)

    def one_plain():
        L.orac_gpu_md_run_async(e1.ctx, 1)

    plain_ms = _timed_steps(one_plain, st1, flush, args.steps)
    if L.orac_gpu_md_collect(e1.ctx):
        raise RuntimeError(L.orac_gpu_last_error(e1.ctx).decode())
    e1.close()
    # the batch
    engines, lams = [], []
    for k in range(nwin):
        e, lam = window_engine(base, k, nwin, device, wl)
        engines.append(e)
        lams.append(lam)
    b = Batch(engines)
    tune_batch = tuned(b)
    stream = torch.cuda.ExternalStream(b.stream(), device=device)
    b.run(args.warmup)
    b.sync()
    cnt = (C.c_int64 * 4)()
    for e in engines:
        e.lib.orac_gpu_counters(e.ctx, cnt, 1)
    step_ms = _timed_steps(lambda: b.run(1, sync=False), stream, flush, args.steps)
    b.sync()
    # pair evaluations of every window over the timed steps (device counters)
    pairs_ewald = pairs_lj = 0
    for e in engines:
        e.lib.orac_gpu_counters(e.ctx, cnt, 0)
        pairs_ewald += int(cnt[2])
        pairs_lj += int(cnt[3])
    # dU/dlambda of every window: energy records written on the device every
    # DUDL_EVERY steps of a batched sampling run after the timed steps
    for e in engines:
        e.md_records(1, reset=True)
    b.run(DUDL_STEPS, energy_every=DUDL_EVERY)
    b.close()
    dudl = []
    for e in engines:
        rec, n = e.md_records(DUDL_STEPS // DUDL_EVERY)
        dudl.append(rec[:, 15].copy())
        e.close()
    st = sorted(step_ms)
    return {"systems": nwin, "atoms_per_window": base.ntap, "total_ms": sum(step_ms),
            "step_ms_p50": st[len(st) // 2], "step_ms_p99": st[min(len(st) - 1, int(0.99 * len(st)))],
            "plain_total_ms": sum(plain_ms), "lambdas": lams, "dudl": dudl, "pairs_ewald": pairs_ewald,
            "pairs_lj": pairs_lj,
            "tuning": {"batch": tune_batch, "plain_window": tune_plain}}


def block_mean_err(x, nblocks=10):
    """Mean and its standard error from the spread of nblocks block means
    (correlated samples of one trajectory)."""
    x = np.asarray(x, dtype=np.float64)
    nb = max(2, min(nblocks, len(x)))
    m = len(x) // nb
    blocks = x[:m * nb].reshape(nb, m).mean(axis=1)
    return float(x.mean()), float(blocks.std(ddof=1) / np.sqrt(nb))


def build_pool(specs):
    """Host-side systems of `specs` (systems.build_spec), built in a spawn
    process pool (no CUDA state is inherited)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    workers = max(1, min(32, (os.cpu_count() or 1), len(specs)))
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(systems.build_spec, specs, chunksize=1))


def uneven_engine(s, spec, device, wl, thermostats=None):
    from orac_b200.engine import Engine

    e = Engine(s, device=device)
    e.set_rem(s.rematom, 0, spec["rem_factor"])  # seg_select kind 0: pairs touching the solute
    if thermostats:
        e.set_thermostat(*thermostats)
    e.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], econst=0.0)
    return e


def uneven_arm(args, wl, device, flush):
    """The uneven HREM batch: args.uneven solvated-chain systems with atom
    counts log-uniform in [3k, 60k] and per-replica solute scaling
    U[0.3, 1.0] (rem_factor on pairs touching the solute), advanced by one
    graph launch per outer step; plain = each system alone on the same
    driver, one after the other."""
    import torch

    from orac_b200.engine import Batch

    specs = systems.uneven_specs(args.uneven)
    t0 = time.perf_counter()
    syst = build_pool(specs)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    engines = [uneven_engine(s, sp, device, wl) for s, sp in zip(syst, specs)]
    t_setup = time.perf_counter() - t0
    footprint = sum(e.footprint() for e in engines)
    kp = max(2, min(args.steps, 5))
    plain_ms = []
    for e in engines:
        L = e.lib
        st = torch.cuda.ExternalStream(L.orac_gpu_get_stream(e.ctx), device=device)
        for _ in range(args.warmup):
            L.orac_gpu_md_run_async(e.ctx, 1)
        if L.orac_gpu_md_collect(e.ctx):
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        ms = _timed_steps(lambda: L.orac_gpu_md_run_async(e.ctx, 1), st, flush, kp)
        if L.orac_gpu_md_collect(e.ctx):
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        plain_ms.append(sum(ms) / len(ms))
    b = Batch(engines)
    tune_batch = tuned(b)
    stream = torch.cuda.ExternalStream(b.stream(), device=device)
    b.run(args.warmup)
    nb = max(3, min(args.steps, 20))
    step_ms = _timed_steps(lambda: b.run(1, sync=False), stream, flush, nb)
    b.sync()
    b.close()
    status = [e.collect() for e in engines]
    for e in engines:
        e.close()
    n = len(engines)
    st = sorted(step_ms)
    bval = ns_per_day(nb * n, wl["dt_h"], sum(step_ms) / 1e3)
    pval = ns_per_day(n, wl["dt_h"], sum(plain_ms) / 1e3)
    nat = [s.ntap for s in syst]
    return {"workload": f"{n} solvated-chain systems, atoms log-uniform in [3k, 60k] ({min(nat)}..{max(nat)}, "
                        f"{sum(nat)} in all), solute 5-10% as 100-atom chains, water at 0.100 atoms/A^3, SPME grid "
                        "about 1 A (32..96), per-replica solute scaling U[0.3, 1.0] as rem_factor (kind 0), "
                        "reciprocal space unscaled, same r-RESPA schedule as the plain workload",
            "systems": n, "value": bval, "unit": "ns/day (aggregate over systems)",
            "ms_per_step": sum(step_ms) / nb, "step_ms_p50": st[len(st) // 2],
            "step_ms_p99": st[min(len(st) - 1, int(0.99 * len(st)))],
            "plain_value": pval, "plain_ms_per_step_sum": sum(plain_ms), "speedup_vs_plain": bval / pval,
            "device_bytes": footprint, "status_ok": all(x == 0 for x in status), "tuning": tune_batch,
            "host_build_s": t_build, "setup_s": t_setup,
            "how": f"one graph launch per H step advances all {n} systems (orac_gpu_batch_run), {nb} timed steps; "
                   f"plain = each system alone, {kp} timed steps each, summed (one at a time)"}


def serve_arm(args, wl, device):
    """The serving loop: Poisson arrivals (20/s, seed 11) over args.serve
    seconds of 500-step segment requests for a population of
    args.serve_systems solvated-chain systems (atoms log-uniform in
    [2k, 100k]), state resident on the device, admission by a 150 GB
    budget, at most 32 segments in flight.  Plain = the same requests one
    at a time, first come first served, each taking 500 x its system's
    measured single-system step time."""
    from orac_b200 import serve

    nsteps = 500
    specs = systems.uneven_specs(args.serve_systems, seed=12, lo=2000, hi=100000, seed_scale=13)
    for sp in specs:
        sp["name"] = sp["name"].replace("uneven", "served")
    syst = build_pool(specs)
    pop = {k: s for k, s in enumerate(syst)}
    # single-system step time of each system (plain path, engine alone)
    t_step = {}
    for k, (s, sp) in enumerate(zip(syst, specs)):
        e = uneven_engine(s.copy(), sp, device, wl)
        L = e.lib
        for _ in range(3):
            L.orac_gpu_md_run_async(e.ctx, 1)
        e.collect()
        t0 = time.perf_counter()
        L.orac_gpu_md_run_async(e.ctx, 10)
        if e.collect():
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        t_step[k] = (time.perf_counter() - t0) / 10
        e.close()
    arrivals = serve.poisson_arrivals(20.0, args.serve, len(specs), seed=11)
    # the plain path run for real on the first requests, one at a time (each
    # system's context built beforehand, as the model assumes): their
    # 500-step service times against the model's 500 x measured step time
    sample = arrivals[:SERVE_PLAIN_SAMPLE]
    measured, modelled = [], []
    for _, sid in sample:
        e = uneven_engine(syst[sid].copy(), specs[sid], device, wl)
        L = e.lib
        for _ in range(3):
            L.orac_gpu_md_run_async(e.ctx, 1)
        e.collect()
        t0 = time.perf_counter()
        L.orac_gpu_md_run_async(e.ctx, nsteps)
        if e.collect():
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        measured.append(time.perf_counter() - t0)
        modelled.append(nsteps * t_step[sid])
        e.close()
    srv = serve.Server(device=device, budget_bytes=150e9, max_active=32, chunk=args.serve_chunk)
    svc = serve.Service(srv, pop, lambda s: uneven_engine(s, specs[int(s.name[len("served"):])], device, wl),
                        nsteps=nsteps)
    # the systems' contexts built and their graphs captured before the
    # arrivals, as the one-at-a-time model takes them (--serve-cold: built
    # on their first request, inside the timed span)
    prewarmed = 0 if args.serve_cold else svc.prewarm()
    res = svc.run(arrivals, timeout=900.0)
    stats = srv.stats()
    svc.close()
    srv.close()
    lat = np.array(sorted(r["latency"] for r in res))
    span = max(r["t_end"] for r in res) - min(r["t_arrival"] for r in res)
    sim_ns = len(res) * nsteps * wl["dt_h"] * 1e-6
    plat, pend = serve.fifo_one_at_a_time(arrivals, [nsteps * t_step[sid] for _, sid in arrivals])
    pspan = pend - arrivals[0][0]
    plat = np.sort(plat)
    nat = [s.ntap for s in syst]

    def pct(a, q):
        return float(a[min(len(a) - 1, int(q * len(a)))])

    return {"workload": f"Poisson arrivals 20/s for {args.serve:g} s ({len(arrivals)} requests) of {nsteps}-step "
                        f"segments, systems drawn from {len(specs)} solvated-chain systems of {min(nat)}..{max(nat)} "
                        "atoms (log-uniform in [2k, 100k], HREM solute scaling), state resident on the device, "
                        "admission by a 150 GB budget, at most 32 segments in flight",
            "requests": len(res), "value": sim_ns / span * 86400.0, "unit": "ns/day (aggregate)",
            "latency_s_p50": pct(lat, 0.5), "latency_s_p99": pct(lat, 0.99),
            "plain_value": sim_ns / pspan * 86400.0, "plain_latency_s_p50": pct(plat, 0.5),
            "plain_latency_s_p99": pct(plat, 0.99),
            "speedup_vs_plain": (sim_ns / span) / (sim_ns / pspan),
            "status_ok": all(r["status"] == 0 for r in res), "builds": svc.builds, "evictions": svc.evictions,
            "prewarmed": prewarmed,
            "peak_reserved_gb": stats["peak_reserved"] / 1e9,
            "plain_check": {"requests": len(sample), "service_s_measured": measured, "service_s_model": modelled,
                            "measured_over_model": sum(measured) / sum(modelled),
                            "how": "the first requests' systems run one at a time through the plain driver, 500 steps "
                                   "each (wall clock, context built beforehand as in the model)"},
            "how": f"native executor (orac_gpu_server_*): per-system streams, {args.serve_chunk} step graphs per chunk, "
                   "pump thread; "
                   "latency = segment end - arrival (host monotonic clock); plain = first-come-first-served single "
                   "server with each request taking 500 x the system's measured single-system step time"}


def f0_arm(args, device, flush):
    """The reference's own test system (F0, test1's schedule and
    parameters, NVE here) through the device-resident driver; its CPU
    restatement on the host cores beside it; ORAC's published rate for the
    same system and schedule (test1) for reference."""
    import torch

    from orac_b200.engine import Engine

    wl = F0_WORKLOAD
    s = wl["build"]()
    k = max(3, min(args.steps, 20))

    def timed(thermos):
        e = Engine(s.copy(), device=device)
        if thermos:
            e.set_thermostat(*thermos)
        e.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], n1respa=wl["n1respa"],
                   n0respa=wl["n0respa"], econst=0.0)
        L = e.lib
        st = torch.cuda.ExternalStream(L.orac_gpu_get_stream(e.ctx), device=device)
        for _ in range(args.warmup):
            L.orac_gpu_md_run_async(e.ctx, 1)
        if e.collect():
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        ms = _timed_steps(lambda: L.orac_gpu_md_run_async(e.ctx, 1), st, flush, k)
        if e.collect():
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        e.close()
        return ms

    ms = timed(None)
    ms_nvt = timed(TEST1_THERMOS)
    val = ns_per_day(k, wl["dt_h"], sum(ms) / 1e3)
    val_nvt = ns_per_day(k, wl["dt_h"], sum(ms_nvt) / 1e3)
    out = {"workload": f"ORAC test1 system as ORAC assembled it (solvated FKBP12 + ligand, {s.ntap} atoms, "
                       f"{len(s.constraints)} bonds to hydrogen rigid, {len(s.bonds)} flexible), SPME alpha 0.37 48^3 "
                       "order 4, shells 5.1/7.8/10.0 A, r-RESPA 15/3/1.5/0.75/0.375 fs, NVE",
           "value": val, "unit": "ns/day", "ms_per_step": sum(ms) / k, "steps": k,
           "orac_published": {"value": TEST1_PUBLISHED_NS_DAY, "unit": "ns/day",
                              "how": "ORAC's own run of this system and schedule (test1/md.out:1061,1063), "
                                     "8 OpenMP threads of an unrecorded CPU, NPT with Nose-Hoover"},
           "speedup_vs_orac_published": val / TEST1_PUBLISHED_NS_DAY,
           "nvt": {"value": val_nvt, "unit": "ns/day", "ms_per_step": sum(ms_nvt) / k,
                   "thermostats": "test1's THERMOS: 298 K, centres of mass, solute and solvent at 10 cm^-1 "
                                  "(ORAC's run adds the ISOSTRESS barostat, not built here)",
                   "speedup_vs_orac_published": val_nvt / TEST1_PUBLISHED_NS_DAY}}
    if not args.no_cpu_baseline:
        t, done, cores = cpu_run(wl, s, 50, 1, budget_s=args.cpu_budget / 2)
        out["cpu_restatement"] = {"value": ns_per_day(done, wl["dt_h"], t), "unit": "ns/day", "cores": cores,
                                  "sample": f"{done} H steps"}
    return out


def hrem_arm(args, wl, device):
    """Hamiltonian replica exchange as ORAC's test2 runs it, batched on one
    GPU: HREM_N replicas of one solvated-chain system (about 20k atoms, a
    70-atom solute chain, the size of test2's ligand + TYR27 segment),
    solute scaling on a geometric ladder from 1 to 0.6 as in test2
    (rem_factor(3) on the pairs touching the solute, seg_select kind 0),
    test2's Nose-Hoover thermostats (298 K, 10 cm^-1; ORAC's run adds the
    barostat), an exchange attempt every 15 steps (60 fs) by ORAC's rule on
    the replicas' segment energies recorded on the device.  Timed by wall
    clock over the exchange intervals (steps, records, decisions and factor
    writes all inside); plain = one replica alone through the same driver."""
    import torch

    from orac_b200 import hrem

    s = systems.solvated_chains(20000, 4242, solute_frac=70 / 20000, name="hrem20k")
    ladder = hrem.ladder_geometric(HREM_N, 0.6)
    kT = units.BOLTZ * TEST1_THERMOS[0] / units.UNITE

    def make(f):
        return uneven_engine(s.copy(), {"rem_factor": float(f)}, device, wl, thermostats=TEST1_THERMOS)

    e1 = make(1.0)
    L = e1.lib
    for _ in range(3):
        L.orac_gpu_md_run_async(e1.ctx, 1)
    e1.collect()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L.orac_gpu_md_run_async(e1.ctx, HREM_EVERY * HREM_INTERVALS)
    if e1.collect():
        raise RuntimeError(L.orac_gpu_last_error(e1.ctx).decode())
    plain_s = time.perf_counter() - t0
    e1.close()
    engines = [make(f) for f in ladder]
    h = hrem.HremBatch(engines, ladder, kT, seed=2)
    tune = tuned(h.batch)
    h.interval(HREM_EVERY)  # warm-up interval (captures the energy-step graphs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(HREM_INTERVALS):
        h.interval(HREM_EVERY)
    secs = time.perf_counter() - t0
    acc = h.acceptance()
    ens = h.ens.tolist()
    h.close()
    status = [e.collect() for e in engines]
    for e in engines:
        e.close()
    steps = HREM_EVERY * HREM_INTERVALS
    val = ns_per_day(steps * HREM_N, wl["dt_h"], secs)
    pval = ns_per_day(steps, wl["dt_h"], plain_s)
    return {"workload": f"{HREM_N} replicas of one solvated-chain system ({s.ntap} atoms, solute {int(s.rematom.sum())} "
                        "atoms), solute scaling 1..0.6 geometric as rem_factor(3) (seg_select kind 0), test2's "
                        "Nose-Hoover thermostats (298 K, 10 cm^-1 each; no barostat), "
                        f"exchange attempts every {HREM_EVERY} steps ({HREM_EVERY * wl['dt_h']:g} fs)",
            "replicas": HREM_N, "value": val, "unit": "ns/day (aggregate over replicas)",
            "plain_value": pval, "speedup_vs_plain": val / pval, "exchanges": HREM_INTERVALS + 1,
            "acceptance_by_pair": [float(a) for a in acc], "final_ensembles": ens,
            "status_ok": all(x == 0 for x in status), "tuning": tune,
            "how": "one graph launch per step advances every replica; each interval ends with an energy step whose "
                   "device record holds the segment energies; ORAC's decision (orac_gpu_rem_exchange) on the host; "
                   "accepted swaps rewrite rem_factor on the device (no graph capture); wall clock over "
                   f"{HREM_INTERVALS} intervals"}


def ne_arm(args, device):
    """The non-equilibrium work swarm of the reference's test4: walkers on
    F0 switch the ligand off along test4's 1.5 ps schedule (charges over
    0.6 ps, then the LJ) with the shifted potential, the lambdas moved and
    the work summed on the device (orac_gpu_md_set_schedule); all walkers
    advance by one graph launch per 15-fs step.  Walkers start from test2's
    three restart states (the states of test4's walkers 1, 2 and 4) with
    their own velocities and with three perturbed copies each (every
    velocity scaled by 1 + 0.01 N(0, 1)).  Timed by wall clock over the
    whole schedule; plain = one walker alone through the same driver."""
    import torch

    from orac_b200.engine import Batch, Engine

    d = np.load(os.path.join(ROOT, "tests", "golden", "ne_test4.npz"))
    sch = d["schedule"]
    wl = NE_WORKLOAD
    nsteps = int(round(1000.0 * sch[-1, 0] / wl["dt_h"]))
    kT = units.BOLTZ * 300.0 / units.UNITE

    def make(k, draw):
        s = f0_test4_system(k)
        if draw:
            rng = np.random.default_rng(1000 * k + draw)
            f = 1.0 + 0.01 * rng.standard_normal(s.ntap)
            s.vx, s.vy, s.vz = s.vx * f, s.vy * f, s.vz * f
        e = Engine(s, device=device)
        e.set_alchemy(s.ss_alchemy, 0.5, 0.5, shifted=True, qshift=4.0, ljshift=0.35)
        e.set_lambda(0.0, 0.0, 0.0, 0.0)
        e.set_schedule(sch[:, 0] * 1000.0, sch[:, 1], sch[:, 2], sch[:, 3], sch[:, 4])
        e.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], n1respa=wl["n1respa"],
                   n0respa=wl["n0respa"])
        return e

    e1 = make(0, 0)
    L = e1.lib
    L.orac_gpu_md_run_async(e1.ctx, 1)  # captures the step graphs
    if e1.collect():
        raise RuntimeError(L.orac_gpu_last_error(e1.ctx).decode())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L.orac_gpu_md_run_async(e1.ctx, nsteps - 1)
    if e1.collect():
        raise RuntimeError(L.orac_gpu_last_error(e1.ctx).decode())
    plain_s = time.perf_counter() - t0
    w_plain = e1.md_work()[0]
    e1.close()
    walkers = [(k, draw) for draw in range(NE_WALKERS // 3) for k in range(3)]
    engines = [make(k, draw) for k, draw in walkers]
    b = Batch(engines)
    tune = tuned(b)
    b.run(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run(nsteps - 1)
    secs = time.perf_counter() - t0
    b.close()
    works = []
    for e in engines:
        works.append(e.md_work()[0] * units.KJMOL)
        if e.collect():
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        e.close()
    works = np.array(works)
    wk = works / (kT * units.KJMOL)
    jar = -kT * units.KJMOL * (np.log(np.mean(np.exp(-(wk - wk.min())))) - wk.min())
    orac_final = {f"walker{w}": float(d[f"wrk{w}"][-1, 5]) for w in (1, 2, 4)}
    val = ns_per_day((nsteps - 1) * len(engines), wl["dt_h"], secs)
    pval = ns_per_day(nsteps - 1, wl["dt_h"], plain_s)
    return {"workload": f"{len(engines)} NE walkers on F0 (14,900 atoms), test4's schedule 15.off "
                        "(1.5 ps: charges off over 0.6 ps, LJ over 0.9 ps), shifted potential 4.0/0.35, shells "
                        "5.0/8.1/12.5 A, SPME 48x49x48, r-RESPA 15/3/1.5/0.75/0.375 fs, NVE",
            "walkers": len(engines), "steps": nsteps, "value": val, "unit": "ns/day (aggregate over walkers)",
            "plain_value": pval, "speedup_vs_plain": val / pval,
            "work_kjmol": [float(x) for x in works],
            "work_same_starts_as_orac": {"walker1": float(works[0]), "walker2": float(works[1]),
                                         "walker4": float(works[2])},
            "orac_printed_final_work_kjmol": orac_final,
            "plain_walker1_work_kjmol": float(w_plain * units.KJMOL),
            "jarzynski_dG_kjmol": float(jar), "mean_work_kjmol": float(works.mean()), "tuning": tune,
            "how": "work per walker summed on the device as ORAC sums it (orac_gpu_md_work); ORAC's final works are "
                   "the last line of test4/PAR000k/1.5.wrk (NPT with thermostats and a COM restraint: the "
                   "trajectories part after ~0.1 ps, so the finals agree only in size); wall clock over the "
                   "schedule after one captured step"}


def config2_arm(args, device, flush):
    """The solvated chain of the second workload: a 1,700-atom bonded chain
    in 7,000 waters (22,700 atoms, 62 A box, SPME 64^3 order 5), FP32 pair
    forces with fixed-point sums, FP64 integration; the chain's bonds,
    bends and torsions on the N0/N1 levels (0.5 fs M step split 2 x 2).
    MD rate of the device-resident driver, and the state's forces and
    energies against the FP64 oracle."""
    import torch

    from orac_b200.engine import Engine

    wl = dict(WORKLOADS["liquid"], n1respa=2, n0respa=2)
    s = systems.config2_polymer()
    e = Engine(s.copy(), device=device)
    e.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], n1respa=wl["n1respa"],
               n0respa=wl["n0respa"], econst=0.0)
    L = e.lib
    st = torch.cuda.ExternalStream(L.orac_gpu_get_stream(e.ctx), device=device)
    for _ in range(args.warmup):
        L.orac_gpu_md_run_async(e.ctx, 1)
    if e.collect():
        raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
    k = max(3, min(args.steps, 20))
    ms = _timed_steps(lambda: L.orac_gpu_md_run_async(e.ctx, 1), st, flush, k)
    if e.collect():
        raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
    x, _ = e.md_state()
    e.close()
    out = {"workload": f"1,700-atom bonded chain in 7,000 waters ({s.ntap} atoms), 62 A box, SPME 64^3 order 5, "
                       "alpha 0.35, shells 5.0/7.5/10.0 A, r-RESPA 4/2/0.5 fs with the chain's bonded terms at "
                       "0.25/0.125 fs, NVE",
           "value": ns_per_day(k, wl["dt_h"], sum(ms) / 1e3), "unit": "ns/day", "ms_per_step": sum(ms) / k,
           "steps": k}
    try:
        out["force_check"] = force_check(s, x)
    except Exception as exc:
        out["force_check"] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def config1_fixed_arm(args, device, flush):
    """The 3,000-water box as specified (31 A, three times liquid density):
    its dynamics heat and stop converging SHAKE within tens of steps, so its
    rate is the force-evaluation rate on a fixed list at the seeded state --
    every shell (M, L, H) and SPME, forces only, device-resident inputs."""
    import ctypes as C

    import torch

    from orac_b200.engine import Engine

    s = systems.config1_water()
    e = Engine(s.copy(), device=device)
    e.update_lists()
    L = e.lib
    dev = torch.device(f"cuda:{device}")
    x = torch.tensor(np.concatenate([s.xp0, s.yp0, s.zp0]), dtype=torch.float64, device=dev)
    g = torch.tensor(np.concatenate(s.group_centres()), dtype=torch.float64, device=dev)
    m = torch.tensor(np.concatenate(s.molecule_centres()), dtype=torch.float64, device=dev)
    f = torch.zeros(3 * s.ntap, dtype=torch.float64, device=dev)
    eer = torch.zeros(1, dtype=torch.float64, device=dev)
    vir = torch.zeros(9, dtype=torch.float64, device=dev)
    st = torch.cuda.ExternalStream(L.orac_gpu_get_stream(e.ctx), device=device)

    def one():
        for sh in "mlh":
            rc = L.orac_gpu_mts_forces_dev(e.ctx, sh.encode(), x.data_ptr(), g.data_ptr(), m.data_ptr(), f.data_ptr(),
                                           None, None)
            if rc:
                raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())
        rc = L.orac_gpu_fft_pme_dev(e.ctx, x.data_ptr(), m.data_ptr(), f.data_ptr(), eer.data_ptr(), vir.data_ptr())
        if rc:
            raise RuntimeError(L.orac_gpu_last_error(e.ctx).decode())

    for _ in range(args.warmup):
        one()
    cnt = (C.c_int64 * 4)()
    L.orac_gpu_counters(e.ctx, cnt, 1)
    k = max(3, min(args.steps, 20))
    ms = _timed_steps(one, st, flush, k)
    L.orac_gpu_counters(e.ctx, cnt, 0)
    e.close()
    secs = sum(ms) / 1e3
    out = {"workload": "3,000 rigid waters in the 31.0 A box as specified (9,000 atoms, 3x liquid density), SPME 32^3 "
                       "order 4, alpha 0.35, shells 5.0/7.5/10.0 A, list fixed at the seeded state",
           "force_evals_per_s": k / secs, "ms_per_force_eval": 1e3 * secs / k,
           "pair_evals_per_s": (cnt[2] + cnt[3]) / secs,
           "how": "one force evaluation = M, L and H shells plus SPME (forces only, device buffers, "
                  "orac_gpu_mts_forces_dev / orac_gpu_fft_pme_dev), CUDA events on the context stream, L2 flushed "
                  "before each"}
    try:
        out["force_check"] = force_check(s, s.cartesian())
    except Exception as exc:
        out["force_check"] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def profile_window_batch(nwin):
    """One batched step of `nwin` lambda windows bracketed for a profiler
    that starts collecting at cudaProfilerStart (the windows' set-up and
    three warm-up steps stay outside)."""
    import torch

    from orac_b200.engine import Batch

    wl = WORKLOADS["liquid"]
    base = systems.ligand_in_water()
    engines = [window_engine(base, k, nwin, 0, wl)[0] for k in range(nwin)]
    b = Batch(engines)
    b.run(3)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    b.run(1)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    b.close()
    for e in engines:
        e.close()
    return 0


def profile_f0(nsteps, thermostats=False):
    """`nsteps` MD steps of the test1 system (F0) bracketed for a profiler
    that starts collecting at cudaProfilerStart (set-up and three warm-up
    steps stay outside); with thermostats, test1's THERMOS."""
    import torch

    from orac_b200.engine import Engine

    wl = F0_WORKLOAD
    e = Engine(wl["build"]().copy())
    if thermostats:
        e.set_thermostat(*TEST1_THERMOS)
    e.md_setup(wl["dt_h"], wl["lrespa"], wl["mrespa"], wl["nupdte"], wl["rshk"], n1respa=wl["n1respa"],
               n0respa=wl["n0respa"], econst=0.0)
    e.md_run(3)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    e.md_run(nsteps)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    rc = e.collect()
    e.close()
    return rc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=6)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    # the 31 A box as specified is three times liquid density: it heats to
    # ~4e4 K within 20 steps and SHAKE stops converging near step 35 in the
    # CPU restatement and the GPU alike, so the MD rate is measured on the
    # same 3,000 waters at liquid density
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="liquid")
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU-baseline sampling")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=64, help="alchemical lambda windows advanced together (0/1: skip)")
    ap.add_argument("--uneven", type=int, default=128, help="systems of the uneven HREM batch (0/1: skip)")
    ap.add_argument("--serve", type=float, default=3.0, help="seconds of Poisson arrivals of the serving leg (0: skip)")
    ap.add_argument("--serve-systems", type=int, default=16, help="systems the serving requests draw from")
    ap.add_argument("--serve-chunk", type=int, default=4, help="captured steps the serving executor queues at a time")
    ap.add_argument("--serve-cold", action="store_true",
                    help="serving leg: build each system's context on its first request instead of before the arrivals")
    ap.add_argument("--no-f0", dest="f0", action="store_false", help="skip the ORAC test1 system leg")
    ap.add_argument("--no-drift", dest="drift", action="store_false", help="skip the 1,000-step energy drift run")
    ap.add_argument("--no-hrem", dest="hrem", action="store_false", help="skip the replica-exchange leg")
    ap.add_argument("--no-ne", dest="ne", action="store_false", help="skip the non-equilibrium work-swarm leg")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the solvated-chain MD leg and the 31 A fixed-list leg")
    ap.add_argument("--profile-window-batch", type=int, default=0, metavar="N",
                    help="profiling aid, no JSON: N lambda windows batched, 3 steps, then one step bracketed by "
                         "cudaProfilerStart/Stop (ncu --profile-from-start off --graph-profiling graph)")
    ap.add_argument("--profile-f0", type=int, default=0, metavar="N",
                    help="profiling aid, no JSON: the test1 system, 3 steps, then N steps bracketed by "
                         "cudaProfilerStart/Stop (ncu --profile-from-start off)")
    ap.add_argument("--profile-thermostats", action="store_true",
                    help="with --profile-f0: test1's Nose-Hoover thermostats (THERMOS 298 K, 10 cm^-1)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.profile_window_batch > 0:
        return profile_window_batch(args.profile_window_batch)
    if args.profile_f0 > 0:
        return profile_f0(args.profile_f0, args.profile_thermostats)
    wl = WORKLOADS[args.workload]
    ws, rank, local = dist_info()
    s = wl["build"]()
    config = {"workload": f"{args.workload}: {wl['desc']}", "atoms": s.ntap, "groups": s.ngrp,
              "step": "one outer r-RESPA step (4 fs)", "l2": "flushed (256 MB write) between timed steps",
              "parallelism": f"replicas x{ws}" if ws > 1 else "single system, 1 GPU"}
    base = {"metric": METRIC, "unit": "ns/day", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32+int64fixed+fp64",
            "data": "synthetic (seeded lattice water, random-orientation, Maxwell-Boltzmann 300 K)",
            "config": config}

    if args.impl == "reference":
        if rank != 0:
            return 0
        t, done, cores = cpu_run(wl, s, args.steps, args.warmup)
        val = ns_per_day(done, wl["dt_h"], t)
        out = dict(base, impl="reference", value=val, ms_per_step=1e3 * t / done,
                   cpu_baseline={"value": val, "unit": "ns/day", "cores": cores, "kind": "port",
                                 "sample": f"{done} H steps of the workload after {args.warmup} warm-up steps "
                                           "(FP64 C restatement of ORAC's loop, OpenMP)"},
                   e2e={"value": val, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        out["steps"] = done
        print(json.dumps(out))
        return 0

    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    res = gpu_arm(args, wl, s, local)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    secs = res["total_ms"] / 1e3
    value = ws * ns_per_day(args.steps, wl["dt_h"], secs)
    peaks = measured_peaks()
    # dominant kernel: the real-space shell kernel (all shells).  It is bound
    # by FP32 issue (LJ + A&S erfc per atom pair, no contraction): the
    # roofline is its pair FLOP rate against the device's measured FP32 FMA
    # rate; the HBM view beside it shows it is far from the memory bound.
    n_l = max(1, res["kpair_n"])
    kp_s = res["kpair_ms"] / 1e3
    npair = res["pairs_ewald"] + res["pairs_lj"]
    flops = 60.0 * res["pairs_ewald"] + 36.0 * res["pairs_lj"]
    fp32 = res.get("fp32_peak")
    fp32_peak_v = fp32 if fp32 else FP32_NOMINAL_TFLOPS
    achieved_tf = flops / kp_s / 1e12 if kp_s > 0 else 0.0
    roofline = {"kernel": "k_pair (real-space r-RESPA shell kernel, all shells)", "bound": "fp32",
                "achieved": achieved_tf, "peak": fp32_peak_v, "unit": "TFLOP/s", "frac": achieved_tf / fp32_peak_v,
                "peak_source": ("measured (FP32 FMA-loop kernel, orac_gpu_fp32_rate, this run)" if fp32
                                else "nominal 148 SM x 128 lanes x 2 x 1.965 GHz"),
                "traffic": ncu_traffic(), "pair_evaluations_per_launch": npair / n_l,
                "flops_per_pair": "60 LJ+Ewald, 36 LJ-only (FMA = 2)", "launches": res["kpair_n"],
                "avg_launch_us": 1e6 * kp_s / n_l, "timing": res["kpair_how"],
                "share_of_step": res["kpair_ms"] / res["total_ms"] if res["total_ms"] else None}
    hbm_peak = peaks.get("hbm_gbs")
    bytes_alg = 12.0 * (res["scanned"] + res["kept"]) + n_l * (40.0 * res["G"] + 48.0 * res["N"])
    achieved_gbs = bytes_alg / kp_s / 1e9 if kp_s > 0 else 0.0
    roofline_hbm = {"kernel": roofline["kernel"], "bound": "hbm", "achieved": achieved_gbs,
                    "peak": hbm_peak if hbm_peak else 6650.0, "unit": "GB/s",
                    "frac": achieved_gbs / (hbm_peak if hbm_peak else 6650.0),
                    "peak_source": "measured" if hbm_peak else "fallback", "traffic": ncu_traffic(),
                    "bytes_per_launch": bytes_alg / n_l,
                    "bytes_counted": "12 B per list entry scanned or kept, 40 B per group, 48 B per atom"}
    rates = {"pair_evals_per_s": npair / (res["total_ms"] / 1e3),
             "shell_evals_per_s": res["shell_evals"] / (res["total_ms"] / 1e3),
             "how": "pair evaluations (non-excluded atom pairs in a shell's band, device counters) and "
                    "real-space shell evaluations (mts_forces calls: 8 M, 2 L, 1 H per 4-fs step) per second "
                    "of the timed steps"}
    cpu = None
    if not args.no_cpu_baseline:
        t, done, cores = cpu_run(wl, s, 200, 1, budget_s=args.cpu_budget)
        cpu = {"value": ns_per_day(done, wl["dt_h"], t), "unit": "ns/day", "cores": cores, "kind": "port",
               "sample": f"{done} H steps of the same workload on {cores} host threads (FP64 C restatement of "
                         "ORAC's r-RESPA loop, OpenMP), after 1 warm-up step"}
    e2e_val = ns_per_day(res["e2e_steps"], wl["dt_h"], res["e2e_s"])
    st = sorted(res["step_ms"])
    out = dict(base, value=value, ms_per_step=res["total_ms"] / args.steps,
               step_ms_p50=st[len(st) // 2], step_ms_p99=st[min(len(st) - 1, int(0.99 * len(st)))],
               roofline=roofline, roofline_hbm=roofline_hbm, force_evals=rates, cpu_baseline=cpu,
               e2e={"value": e2e_val, "unit": "ns/day", "h2d_bytes_per_step": res["bytes_io"],
                    "d2h_bytes_per_step": res["bytes_io"],
                    "how": "orac_gpu_md_set_state (pinned host -> device), one step, orac_gpu_md_get_state "
                           "(device -> pinned host, with the status flags), orac_gpu_md_collect, wall clock"},
               gpu_launches=res["launches"], clocks=res["clocks"], tuning=res["tuning"])
    for key in ("force_check", "energy_conservation", "step_breakdown", "nvt"):
        if key in res:
            out[key] = res[key]
    if "batched" in res:
        bt = res["batched"]
        bval = ns_per_day(args.steps, wl["dt_h"], bt["total_ms"] / 1e3) * bt["systems"]
        pval = ns_per_day(args.steps, wl["dt_h"], bt["plain_total_ms"] / 1e3)
        stats = [block_mean_err(x) for x in bt["dudl"]]
        mean = np.array([m for m, _ in stats]) * units.KJMOL
        err = np.array([e for _, e in stats]) * units.KJMOL
        lam = np.asarray(bt["lambdas"])
        wts = np.gradient(lam) * 0.0  # trapezoid weights
        wts[1:] += 0.5 * np.diff(lam)
        wts[:-1] += 0.5 * np.diff(lam)
        # the pair kernel's FP32 rate with the device full: every window's
        # pair FLOPs over the whole batched step time (the step also runs
        # SPME, drifts and the bonded levels, so this bounds k_pair's rate
        # from below)
        bflop = 60.0 * bt["pairs_ewald"] + 36.0 * bt["pairs_lj"]
        btf = bflop / (bt["total_ms"] / 1e3) / 1e12
        device_full = {"pair_evals_per_s": (bt["pairs_ewald"] + bt["pairs_lj"]) / (bt["total_ms"] / 1e3),
                       "achieved_tflops": btf, "peak_tflops": roofline.get("peak"),
                       "frac_of_fp32": btf / roofline["peak"] if roofline.get("peak") else None,
                       "how": "pair FLOPs of all windows (60 per LJ+Ewald pair, 36 per LJ-only pair, device "
                              "counters) over the whole batched step time, against the same measured FP32 FMA rate "
                              "as roofline: a lower bound on k_pair's own rate with the device full"}
        out["batched"] = {
            "workload": f"{bt['systems']} alchemical lambda windows (lambda_k = k/{bt['systems'] - 1}, charges "
                        "then LJ switched off) of a 40-atom "
                        f"flexible ligand in the liquid water box ({bt['atoms_per_window']} atoms per window), "
                        "soft-core force_alchemy, SPME of the scaled charges, bonded N0/N1 levels",
            "systems": bt["systems"], "value": bval, "unit": "ns/day (aggregate over windows)",
            "ms_per_step": bt["total_ms"] / args.steps, "step_ms_p50": bt["step_ms_p50"],
            "step_ms_p99": bt["step_ms_p99"], "plain_window_value": pval,
            "speedup_vs_plain": bval / pval,
            "dudl_kjmol": {"lambda": [round(float(x), 5) for x in lam], "mean": [float(x) for x in mean],
                           "stderr": [float(x) for x in err], "samples_per_window": len(bt["dudl"][0]),
                           "trapezoid_dG": float((wts * mean).sum()),
                           "trapezoid_dG_stderr": float(np.sqrt(((wts * err) ** 2).sum())),
                           "how": f"energy records on the device every {DUDL_EVERY} steps of a batched run of "
                                  f"{DUDL_STEPS} steps (orac_gpu_batch_run_energy) after the timed steps; mean and "
                                  "standard error from 10 block means per window",
                           "note": "lambda in [0, 0.5] switches the ligand's charges off (lrmq = 2 lambda), "
                                   "[0.5, 1] its LJ (lrm = 2 lambda - 1), ORAC's NE order; each window starts "
                                   "from the same unequilibrated state and samples a few ps, so the sum is a "
                                   "short-run estimate, not a converged free energy"},
            "tuning": bt["tuning"],
            "device_full": device_full,
            "how": "one graph launch per H step advances every window (orac_gpu_batch_run); plain = one window "
                   "alone through the same driver; both with the real-space kernel's launch configuration chosen by "
                   "the autotuner (orac_gpu_batch_tune / orac_gpu_tune)"}
    elif "batched_error" in res:
        out["batched"] = {"error": res["batched_error"]}
    for key in ("orac_test1", "config2", "config1_as_specified", "hrem", "ne_swarm", "uneven", "served"):
        if key in res:
            out[key] = res[key]
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
