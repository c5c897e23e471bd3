"""Host-side mirror of ORAC's nonbonded force-path interface over
liborac_gpu.so.

`Engine` owns one GPU context for one System and exposes the reference's
routine names with their argument meaning: mts_forces (per r-RESPA shell),
lc_list, fft_pme, do_pmesh_kspace, fnb14, fnbgrp, ferrf, cself.  update_lists
and refresh_m_list replay the driver's list-update sequence of
src/mtsmd.f:2403-2470 and :3287-3295, including its temporary swaps of the
shell radii (done here through orac_gpu_set_shells).  Every call goes through
the C ABI with host arrays, exactly as a Fortran caller would.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import lib as L
from .lib import check, colmajor, f64, i32


class Engine:
    def __init__(self, s, device=0):
        self.s = s
        self.lib = L.load()
        ctx = C.c_void_p()
        rc = self.lib.orac_gpu_create(device, C.byref(ctx))
        if rc != L.ORAC_OK:
            raise L.OracGpuError(f"orac_gpu_create: {L.ERRORS.get(rc, rc)}")
        self.ctx = ctx
        self._upload()

    def close(self):
        if self.ctx:
            self.lib.orac_gpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ setup
    def _upload(self):
        s = self.s
        self._type_cm = i32(np.asarray(s.type_table).T.ravel())
        check(self.ctx, self.lib.orac_gpu_set_topology(
            self.ctx, s.ntap, s.ngrp, s.nprot, i32(s.grppt.ravel()), i32(s.atomp), i32(s.atomg), i32(s.ss_index),
            f64(s.charge), i32(s.nbtype), s.ntype, self._type_cm, f64(s.ecc12), f64(s.ecc6), f64(s.mass),
            f64(s.pmass), s.massinfty, i32(s.mapnl), len(s.mapnl)), "set_topology")
        n1, n2, n3 = s.nfft
        check(self.ctx, self.lib.orac_gpu_set_ewald(self.ctx, 1, s.alphal, s.order, n1, n2, n3, s.rkcut),
              "set_ewald")
        self.set_shells(s.shells)
        if s.ncell is not None:
            check(self.ctx, self.lib.orac_gpu_set_linked_cell(self.ctx, *s.ncell), "set_linked_cell")
        else:
            check(self.ctx, self.lib.orac_gpu_set_linked_cell(self.ctx, 0, 0, 0), "set_linked_cell")
        self.set_box(s.co)
        self._coords()
        if s.has_intra():
            self._upload_intra()

    def _upload_intra(self):
        """Bonded terms and intramolecular pair lists (orac_gpu_set_bonded,
        orac_gpu_set_intra_pairs)."""
        s = self.s
        a = s.intra_lists()
        self._intra = a
        check(self.ctx, self.lib.orac_gpu_set_bonded(
            self.ctx, len(a["lbnd"]) // 2, a["lbnd"], a["r0"], a["kb"], len(a["lbndg"]) // 3, a["lbndg"],
            a["bendpot"], len(a["ltor"]) // 4, a["ltor"], a["tpota"], a["tpotb"], len(a["litr"]) // 4, a["litr"],
            a["ipota"], a["ipotb"], a["ipotc"]), "set_bonded")
        check(self.ctx, self.lib.orac_gpu_set_intra_pairs(
            self.ctx, len(a["int14"]) // 2, a["int14"], a["type14"], a["ecc1412"], a["ecc146"], len(a["ecc1412"]),
            s.fudge, 1.0, len(a["ingrp"]) // 2, a["ingrp"], len(a["int13"]) // 2, a["int13"]), "set_intra_pairs")

    def intra_n0(self):
        """mts_intra_n0: (F (3,N), energies[6])."""
        r = self.s.cartesian()
        F = [np.zeros(self.s.ntap) for _ in range(3)]
        e = np.zeros(6)
        check(self.ctx, self.lib.orac_gpu_mts_intra_n0(self.ctx, f64(r[0]), f64(r[1]), f64(r[2]), *F, e), "intra_n0")
        return np.stack(F), e

    def intra_n1(self):
        """mts_intra_n1: (F (3,N), energies[10])."""
        r = self.s.cartesian()
        F = [np.zeros(self.s.ntap) for _ in range(3)]
        e = np.zeros(10)
        check(self.ctx, self.lib.orac_gpu_mts_intra_n1(self.ctx, f64(r[0]), f64(r[1]), f64(r[2]), *F, e), "intra_n1")
        return np.stack(F), e

    def set_shells(self, sh):
        check(self.ctx, self.lib.orac_gpu_set_shells(self.ctx, sh.rcutm, sh.rtolm, sh.rneim, sh.rcutl, sh.rtoll,
                                                     sh.rneil, sh.rcuth, sh.rtolh, sh.rneih), "set_shells")

    def set_box(self, co):
        self.s.co = np.asarray(co, dtype=np.float64)
        check(self.ctx, self.lib.orac_gpu_set_box(self.ctx, colmajor(self.s.co), colmajor(np.linalg.inv(self.s.co))),
              "set_box")

    def _coords(self):
        s = self.s
        self.xp0, self.yp0, self.zp0 = f64(s.xp0), f64(s.yp0), f64(s.zp0)
        xg, yg, zg = s.group_centres()
        self.xpg, self.ypg, self.zpg = f64(xg), f64(yg), f64(zg)
        xm, ym, zm = s.molecule_centres()
        self.xpcm, self.ypcm, self.zpcm = f64(xm), f64(ym), f64(zm)

    def set_coords(self, xp0, yp0, zp0):
        self.s.xp0, self.s.yp0, self.s.zp0 = f64(xp0), f64(yp0), f64(zp0)
        self._coords()

    # ------------------------------------------------------------ lists
    def lc_list(self, rcut):
        n = C.c_int64()
        check(self.ctx, self.lib.orac_gpu_lc_list(self.ctx, rcut, self.xpg, self.ypg, self.zpg, C.byref(n)),
              "lc_list")
        return int(n.value)

    def mts_forces(self, rshell, nstep=0):
        """One mts_forces call: returns (F (3,N), energies dict, stress (3,3))."""
        s = self.s
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        st = np.zeros(9)
        e = [C.c_double() for _ in range(8)]
        check(self.ctx, self.lib.orac_gpu_mts_forces(
            self.ctx, nstep, rshell.encode(), self.xp0, self.yp0, self.zp0, self.xpg, self.ypg, self.zpg, self.xpcm,
            self.ypcm, self.zpcm, *[C.byref(x) for x in e], fx, fy, fz, st), f"mts_forces('{rshell}')")
        names = ["ucns", "ucos", "virs", "virsp", "ucnp", "ucop", "ucnsp", "ucosp"]
        en = {k: v.value for k, v in zip(names, e)}
        return np.stack([fx, fy, fz]), en, st.reshape(3, 3, order="F")

    @staticmethod
    def ue6(en):
        """Energies in the oracle's order: LJ slt, slv, mixed; Coulomb slt, slv, mixed."""
        return np.array([en["ucnp"], en["ucns"], en["ucnsp"], en["ucop"], en["ucos"], en["ucosp"]])

    # ------------------------------------------------------ variants
    def set_rem(self, rematom, kind=0, factor=1.0):
        """force_rem for every later shell (orac_gpu_set_rem); None: standard."""
        arr = None if rematom is None else i32(np.asarray(rematom) != 0)
        check(self.ctx, self.lib.orac_gpu_set_rem(self.ctx, arr, int(kind), float(factor)), "set_rem")

    def set_alchemy(self, ss_alchemy, qsoft=0.5, ljsoft=0.5, opls=False, shifted=False, qshift=0.0, ljshift=0.0):
        """force_alchemy with ORAC's per-atom soft-core parameters, or with
        `shifted` force_ALCHEMY_shift (SHIFT-POT qshift ljshift); None:
        standard."""
        if ss_alchemy is None:
            check(self.ctx, self.lib.orac_gpu_set_alchemy(self.ctx, None, None, None, 0.0, 0.0, 0), "set_alchemy")
            return
        rmin, epsm = self.s.alchemy_params()
        check(self.ctx, self.lib.orac_gpu_set_alchemy(self.ctx, i32(ss_alchemy), f64(rmin), f64(epsm), qsoft, ljsoft,
                                                      int(opls)), "set_alchemy")
        check(self.ctx, self.lib.orac_gpu_set_alchemy_shift(self.ctx, int(bool(shifted)), float(qshift),
                                                            float(ljshift)), "set_alchemy_shift")

    def set_lambda(self, ladd, lrm, laddq, lrmq, ladd0=None, lrm0=None, laddq0=None, lrmq0=None, intramol=False,
                   ljintra=False, dlam=None):
        """cpropar lambdas (previous ones default to the current); dlam =
        d(ladd, lrm, laddq, lrmq)/dlambda for the dU/dlambda output."""
        lam = [ladd, lrm, laddq, lrmq, ladd if ladd0 is None else ladd0, lrm if lrm0 is None else lrm0,
               laddq if laddq0 is None else laddq0, lrmq if lrmq0 is None else lrmq0]
        d = None if dlam is None else f64(dlam)
        check(self.ctx, self.lib.orac_gpu_set_lambda(self.ctx, f64(lam), int(intramol), int(ljintra),
                                                     None if d is None else d.ctypes.data), "set_lambda")

    def variant_energies(self):
        """(seg_ene, dwrk, U0 LJ, U0 Coulomb, dU/dlambda, PME work, PME
        dU/dlambda, self dU/dlambda) of the last energy evaluations
        (orac_gpu_variant_energies)."""
        out = np.zeros(8)
        check(self.ctx, self.lib.orac_gpu_variant_energies(self.ctx, out), "variant_energies")
        return out

    def update_lists(self):
        """H list by linked cells (or the 'u' all-pairs update), then the two
        phony calls deriving the L and M lists (src/mtsmd.f:2403-2470)."""
        sh = self.s.shells
        if self.s.ncell is None:
            self.mts_forces("u")
        else:
            self.lc_list(sh.rcuth + sh.rtolh + sh.rneih)
        sh1 = dataclasses.replace(sh, rcuth=sh.rcutl, rtolh=0.0)
        self.set_shells(sh1)
        self.mts_forces("h")
        sh2 = dataclasses.replace(sh1, rcutl=sh.rcutm, rtoll=0.0)
        self.set_shells(sh2)
        self.mts_forces("l")
        self.set_shells(sh)

    def shell(self, rshell):
        return self.mts_forces(rshell)

    def refresh_m_list(self):
        sh = self.s.shells
        self.set_shells(dataclasses.replace(sh, rcutl=sh.rcutm))
        self.mts_forces("l")
        self.set_shells(sh)

    def list_pairs(self):
        lp = (C.c_int64 * 3)()
        n = C.c_int64()
        check(self.ctx, self.lib.orac_gpu_stats(self.ctx, lp, C.byref(n)), "stats")
        return {"h": lp[0], "l": lp[1], "m": lp[2]}, n.value

    # -------------------------------------------------------------- PME
    def fft_pme(self, pressure=True):
        s = self.s
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        st = np.zeros(9)
        eer = C.c_double()
        check(self.ctx, self.lib.orac_gpu_fft_pme(self.ctx, self.xp0, self.yp0, self.zp0, self.xpcm, self.ypcm,
                                                  self.zpcm, C.byref(eer), fx, fy, fz, st, int(pressure)), "fft_pme")
        return np.stack([fx, fy, fz]), eer.value, st.reshape(3, 3, order="F")

    def do_pmesh_kspace(self, x, y, z, charge, recip, volume, alpha, order, nfft):
        n = len(x)
        dx = np.zeros(n)
        dy = np.zeros(n)
        dz = np.zeros(n)
        vir = np.zeros(9)
        eer = C.c_double()
        check(self.ctx, self.lib.orac_gpu_do_pmesh_kspace(self.ctx, n, f64(x), f64(y), f64(z), f64(charge),
                                                          colmajor(recip), volume, alpha, order, nfft[0], nfft[1],
                                                          nfft[2], C.byref(eer), dx, dy, dz, vir), "do_pmesh_kspace")
        return np.stack([dx, dy, dz]), eer.value, vir.reshape(3, 3, order="F")

    # ------------------------------------------------------ short lists
    def _cart(self):
        r = self.s.cartesian()
        return f64(r[0]), f64(r[1]), f64(r[2])

    def fnb14(self, cut=True):
        s = self.s
        x, y, z = self._cart()
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        ue = np.zeros(4)
        check(self.ctx, self.lib.orac_gpu_fnb14(self.ctx, x, y, z, int(cut), i32(s.int14.ravel()), len(s.int14),
                                                i32(s.type14), f64(s.ecc1412), f64(s.ecc146), len(s.ecc1412),
                                                s.fudge, 1.0, fx, fy, fz, ue), "fnb14")
        return np.stack([fx, fy, fz]), ue

    def fnbgrp(self):
        s = self.s
        x, y, z = self._cart()
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        ue = np.zeros(4)
        check(self.ctx, self.lib.orac_gpu_fnbgrp(self.ctx, x, y, z, i32(s.ingrp.ravel()), len(s.ingrp), fx, fy, fz,
                                                 ue), "fnbgrp")
        return np.stack([fx, fy, fz]), ue

    def ferrf(self, pairs, fudge, iz=1):
        s = self.s
        x, y, z = self._cart()
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        fs = np.zeros(2)
        p = i32(np.asarray(pairs).reshape(-1, 2).ravel())
        check(self.ctx, self.lib.orac_gpu_ferrf(self.ctx, fudge, x, y, z, iz, p, len(p) // 2, fs, fx, fy, fz),
              "ferrf")
        return np.stack([fx, fy, fz]), fs

    # --------------------------------------------------------------- MD
    def md_setup(self, dt_h, lrespa, mrespa, nupdte, rshk="l", n1respa=1, n0respa=1, econst=0.0, graphs=True):
        """Device-resident r-RESPA run of this system (orac_gpu_md_setup)."""
        s = self.s
        r = s.xyz_restart if s.xyz_restart is not None else s.cartesian()
        self._cn = i32(s.constraints.ravel())
        self._dss = f64(s.cdist ** 2)
        check(self.ctx, self.lib.orac_gpu_md_setup(self.ctx, f64(r[0]), f64(r[1]), f64(r[2]), f64(s.vx), f64(s.vy),
                                                   f64(s.vz), self._cn, self._dss, len(s.constraints), dt_h, lrespa,
                                                   mrespa, n1respa, n0respa, nupdte, rshk.encode(), econst),
              "md_setup")
        check(self.ctx, self.lib.orac_gpu_md_set_graphs(self.ctx, int(graphs)), "md_set_graphs")

    MD_REC = 16  # doubles per energy record (ORAC_MD_REC)

    def md_run(self, nsteps, energy_every=0):
        """nsteps outer steps; every energy_every steps a record of MD_REC
        doubles: step, kinetic, (LJ, Coulomb) of M, L, H, SPME, constant,
        total, flags, bonded, 1-4 + intra-group, erf corrections, 0."""
        R = self.MD_REC
        nrec = nsteps // energy_every if energy_every else 0
        rec = np.zeros(max(1, nrec) * R)
        check(self.ctx, self.lib.orac_gpu_md_run(self.ctx, nsteps, energy_every, rec), "md_run")
        return rec[:nrec * R].reshape(-1, R)

    def set_rem_factor_async(self, factor, stream=None):
        """A new rem_factor(3), in stream order (orac_gpu_set_rem_factor_async)."""
        check(self.ctx, self.lib.orac_gpu_set_rem_factor_async(self.ctx, float(factor), stream), "set_rem_factor_async")

    def set_pair_tuning(self, lpg_m=0, lpg_lh=0, minb=0):
        """Launch configuration of the real-space kernel (0: the mode's default)."""
        check(self.ctx, self.lib.orac_gpu_set_pair_tuning(self.ctx, lpg_m, lpg_lh, minb), "set_pair_tuning")

    def pair_tuning(self):
        out = (C.c_int * 3)()
        check(self.ctx, self.lib.orac_gpu_get_pair_tuning(self.ctx, out), "get_pair_tuning")
        return tuple(out)

    def tune(self, trial=6, cache=None, force=False):
        """Autotune the real-space kernel on this context's MD steps
        (orac_gpu_tune): ((lpg_m, lpg_lh, minb), ms per step)."""
        out = (C.c_int * 3)()
        ms = C.c_double()
        path = cache.encode() if cache else None
        check(self.ctx, self.lib.orac_gpu_tune(self.ctx, trial, path, int(force), out, C.byref(ms)), "tune")
        return tuple(out), ms.value

    def md_records(self, max_records=2048, reset=False):
        """The energy records kept on the device (orac_gpu_md_records): the
        newest up to max_records, oldest first, and the number written."""
        R = self.MD_REC
        out = np.zeros(max(1, max_records) * R)
        n = C.c_int64()
        check(self.ctx, self.lib.orac_gpu_md_records(self.ctx, max_records, out.ctypes.data, C.byref(n),
                                                     int(reset)), "md_records")
        k = min(n.value, max_records, 2048)
        return out[:k * R].reshape(-1, R), n.value

    def set_schedule(self, times_fs, ladded, laddedq, lremoved, lremovedq, t0=0.0, ljintra=False):
        """A non-equilibrium alchemical run (orac_gpu_md_set_schedule): the
        lambdas follow the schedule from t0 (fs) on; before md_setup."""
        sch = [f64(times_fs), f64(ladded), f64(laddedq), f64(lremoved), f64(lremovedq)]
        self._schedule = sch
        check(self.ctx, self.lib.orac_gpu_md_set_schedule(self.ctx, len(sch[0]), *[a.ctypes.data for a in sch],
                                                          float(t0), int(ljintra)), "md_set_schedule")

    def md_work(self):
        """(work, rtime, (ladd, lrm, laddq, lrmq), held terms[8]) of the
        schedule's run (orac_gpu_md_work); work in internal energy units."""
        out = np.zeros(14)
        check(self.ctx, self.lib.orac_gpu_md_work(self.ctx, out.ctypes.data), "md_work")
        return float(out[0]), float(out[1]), tuple(out[2:6]), out[6:14].copy()

    def set_thermostat(self, temp, nu_com, nu_solute, nu_solvent):
        """ORAC's THERMOS (orac_gpu_md_set_thermostat): Nose-Hoover
        thermostats of the molecular centres of mass, the solute and the
        solvent at temp (K), frequencies in cm^-1; before md_setup."""
        check(self.ctx, self.lib.orac_gpu_md_set_thermostat(self.ctx, float(temp), float(nu_com), float(nu_solute),
                                                            float(nu_solvent)), "md_set_thermostat")

    def md_thermostat(self):
        """(eta[3], etap[3], Q[3], ndf[3], energy) of the three thermostats."""
        out = np.zeros(13)
        check(self.ctx, self.lib.orac_gpu_md_thermostat(self.ctx, out.ctypes.data), "md_thermostat")
        return out[0:3].copy(), out[3:6].copy(), out[6:9].copy(), out[9:12].astype(int), float(out[12])

    def set_thermostat_state(self, eta, etap):
        """A restart's thermostat coordinates and velocities
        (orac_gpu_md_set_thermostat_state); after md_setup."""
        e, p = f64(eta), f64(etap)
        check(self.ctx, self.lib.orac_gpu_md_set_thermostat_state(self.ctx, e.ctypes.data, p.ctypes.data),
              "md_set_thermostat_state")

    def md_work_trace(self, max_records=8192):
        """(rtime, work) after each M step, oldest first, and the count."""
        out = np.zeros(2 * max(1, max_records))
        n = C.c_int64()
        check(self.ctx, self.lib.orac_gpu_md_work_trace(self.ctx, max_records, out.ctypes.data, C.byref(n)),
              "md_work_trace")
        k = min(n.value, max_records, 8192)
        return out[:2 * k].reshape(-1, 2), n.value

    def md_state(self):
        n = self.s.ntap
        a = [np.zeros(n) for _ in range(6)]
        check(self.ctx, self.lib.orac_gpu_md_get_state(self.ctx, *a), "md_get_state")
        return np.stack(a[:3]), np.stack(a[3:])

    def footprint(self):
        """Bytes of device memory the context holds (orac_gpu_footprint)."""
        b = C.c_int64(0)
        check(self.ctx, self.lib.orac_gpu_footprint(self.ctx, C.byref(b)), "footprint")
        return b.value

    def collect(self):
        """Wait for queued steps and return the run's status code
        (orac_gpu_md_collect: SHAKE convergence, list capacity)."""
        return self.lib.orac_gpu_md_collect(self.ctx)

    def cself(self):
        a = C.c_double()
        b = C.c_double()
        check(self.ctx, self.lib.orac_gpu_cself(self.ctx, self.s.rkcut, C.byref(a), C.byref(b)), "cself")
        return a.value, b.value


class Batch:
    """Many Engines advanced together by one graph launch per H step
    (orac_gpu_batch_*).  Every engine must have run md_setup."""

    def __init__(self, engines):
        self.engines = list(engines)
        self.lib = L.load()
        arr = (C.c_void_p * len(self.engines))(*[e.ctx.value for e in self.engines])
        h = C.c_void_p()
        rc = self.lib.orac_gpu_batch_create(arr, len(self.engines), C.byref(h))
        if rc != L.ORAC_OK:
            msg = self.lib.orac_gpu_batch_last_error(h).decode() if h.value else ""
            if h.value:
                self.lib.orac_gpu_batch_destroy(h)
            raise L.OracGpuError(f"orac_gpu_batch_create: {L.ERRORS.get(rc, rc)} {msg}")
        self.h = h

    def _check(self, rc, what):
        if rc != L.ORAC_OK:
            raise L.OracGpuError(f"{what}: {L.ERRORS.get(rc, rc)} {self.lib.orac_gpu_batch_last_error(self.h).decode()}")

    def run(self, nsteps, sync=True, energy_every=0):
        """nsteps H steps of every system; with energy_every > 0 every
        energy_every-th step writes each system's energy record."""
        if energy_every:
            self._check(self.lib.orac_gpu_batch_run_energy(self.h, nsteps, energy_every), "batch_run_energy")
        else:
            self._check(self.lib.orac_gpu_batch_run(self.h, nsteps), "batch_run")
        if sync:
            self.sync()

    def sync(self):
        self._check(self.lib.orac_gpu_batch_sync(self.h), "batch_sync")

    def set_rem_factors(self, factors):
        """Every member's rem_factor(3), on the batch's stream
        (orac_gpu_batch_set_rem_factors)."""
        self._check(self.lib.orac_gpu_batch_set_rem_factors(self.h, np.ascontiguousarray(factors, dtype=np.float64)),
                    "batch_set_rem_factors")

    def tune(self, trial=6, cache=None, force=False):
        """Autotune the real-space kernel on the batched steps
        (orac_gpu_batch_tune): ((lpg_m, lpg_lh, minb), ms per batched step)."""
        out = (C.c_int * 3)()
        ms = C.c_double()
        path = cache.encode() if cache else None
        self._check(self.lib.orac_gpu_batch_tune(self.h, trial, path, int(force), out, C.byref(ms)), "batch_tune")
        return tuple(out), ms.value

    def stream(self):
        return self.lib.orac_gpu_batch_stream(self.h)

    def close(self):
        if self.h:
            self.lib.orac_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
