"""ORACLE — test infrastructure only.

ctypes front end of liborac_oracle.so (the FP64 CPU restatement of ORAC's
nonbonded force path).  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module, as the checker.  Parity status: pinned
on the energy records and the NE work ORAC printed for its own test system
(see orac_oracle.h).

The Oracle class drives the restated routines in the order ORAC's r-RESPA
driver does (src/mtsmd.f:2403-2470 for the list update, :3030/:3185/:3263 for
the shell evaluations, :3287-3295 for the phony M-list refresh).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborac_oracle.so")

_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_erfc_as.restype = C.c_double
        L.orc_erfc_as.argtypes = [C.c_double]
        L.orc_decide_force.restype = C.c_int
        L.orc_decide_force.argtypes = [C.c_double, C.c_double]
        L.orc_lc_index.restype = C.c_int
        L.orc_lc_index.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _D, _I, _I, _I]
        L.orc_lc_list.restype = C.c_long
        L.orc_lc_list.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _I, C.c_double, _D, _D, _D, _D,
                                  C.c_int, _I, C.c_long]
        L.orc_force.restype = C.c_long
        L.orc_force.argtypes = [_I, _D, _D, _D, _D, _D, _D, _D, _I, _I, C.c_int, C.c_int, _I, _D, _D, _D, _I, _D,
                                _D, _D, C.c_double, _I, C.c_int, _I, _D, _D, _D, _D, _D, _I, _I, C.c_long,
                                C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _D, C.c_int, _D,
                                C.c_double, C.c_int, C.c_int, C.c_int]
        L.orc_force_ex.restype = C.c_long
        L.orc_force_ex.argtypes = L.orc_force.argtypes + [C.POINTER(Variant), _D]
        L.orc_alch_set.argtypes = [C.POINTER(C.c_double * 18), C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
        L.orc_fpbond.argtypes = [_I, _I, C.c_int, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        L.orc_fpbend.argtypes = [_I, _I, C.c_int, _D, _D, _D, _D, _D, _D, _D, _D]
        L.orc_fptors.restype = C.c_int
        L.orc_fptors.argtypes = [_I, _I, C.c_int, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        L.orc_fitors.restype = C.c_int
        L.orc_fitors.argtypes = [_I, _I, C.c_int, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        L.orc_load_bsp_moduli.argtypes = [_D, _D, _D, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_fill_bspline.argtypes = [C.c_double, C.c_int, _D, _D]
        L.orc_fft1d.argtypes = [C.c_int, _D, C.c_int]
        L.orc_fft3d_r2c.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D]
        L.orc_fft3d_c2r.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D]
        L.orc_scalar_sum.argtypes = [_D, C.c_double, C.c_double, _D, _D, _D, _D, C.c_int, C.c_int, C.c_int, _D,
                                     _D, C.c_double]
        L.orc_do_pmesh_kspace.argtypes = [C.c_int, _D, _D, _D, _D, _D, C.c_double, C.c_double, C.c_int, C.c_int,
                                          C.c_int, C.c_int, _D, _D, _D, _D, _D, C.c_double, C.c_int]
        L.orc_fft_pme.argtypes = [C.c_int, _D, _D, _D, _D, _D, _D, _D, _D, _D, C.c_double, C.c_double, C.c_int,
                                  C.c_int, C.c_int, C.c_int, _D, _D, _D, _D, _D, _I, C.c_int, C.c_double, C.c_int]
        L.orc_ferrf.argtypes = [_I, C.c_double, _D, C.c_double, _D, _D, _D, C.c_int, _I, C.c_int, _D, _D, _D, _D]
        L.orc_cself.argtypes = [_I, _D, C.c_int, C.c_double, C.c_double, _D, _D]
        L.orc_fnb14.argtypes = [_I, _D, _D, _D, _D, C.c_int, _D, _D, C.c_int, C.c_int, C.c_double, _I, C.c_int,
                                _I, C.c_double, C.c_double, _D, _D, _D, _D]
        L.orc_fnbgrp.argtypes = [_I, _D, _D, _D, _D, _I, _D, _D, C.c_int, C.c_double, _I, C.c_int, _D, _D, _D, _D]
        L.orc_alch_atom_lambdas.argtypes = [C.c_int, _I, C.c_double, C.c_double, _D]
        L.orc_alch_listqq.restype = C.c_int
        L.orc_alch_listqq.argtypes = [C.c_int, _I, _I, C.c_int, _I, C.c_int]
        L.orc_ferrf_alchemy_add.argtypes = [_I, C.c_double, _D, _D, _D, _D, _D, _D, _I, C.c_int, C.c_int, _D, _D,
                                            _D, _D, _D]
        L.orc_fnb14_alchemy.argtypes = [_I, _D, _D, _D, _D, _D, _D, C.c_double, _I, C.c_int, _I, C.c_double,
                                        C.c_double, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        _lib = L
    return _lib


class Variant(C.Structure):
    """orc_variant (orac_oracle.h): REM segment or soft-core alchemy."""

    _fields_ = [("mode", C.c_int), ("rematom", C.c_void_p), ("rem_kind", C.c_int), ("rem_factor", C.c_double),
                ("ss_alchemy", C.c_void_p), ("rmin", C.c_void_p), ("epsm", C.c_void_p), ("qsoft", C.c_double),
                ("ljsoft", C.c_double), ("opls", C.c_int), ("fact", C.c_double * 18), ("factq", C.c_double * 18),
                ("fact0", C.c_double * 18), ("factq0", C.c_double * 18), ("shifted", C.c_int),
                ("qshift", C.c_double), ("ljshift", C.c_double)]


def alch_set(ladd, lrm, intramol=False, ljintra=False, qq=False):
    """alch_set (src/force_alchemy_shifted.f:732-790) as a (2, 9) table
    [k, t + 4]."""
    t = (C.c_double * 18)()
    lib().orc_alch_set(C.byref(t), ladd, lrm, int(intramol), int(ljintra), int(qq))
    return np.array(t[:]).reshape(2, 9)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def intra_lists(s):
    """Flat lists of the intramolecular terms (System.intra_lists)."""
    return {k: (_i(v) if v.dtype.kind == "i" else _f(v)) for k, v in s.intra_lists().items()}


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _colmajor(m):
    return np.ascontiguousarray(np.asarray(m, dtype=np.float64).T).ravel()


def default_threads():
    return max(1, os.cpu_count() or 1)


class Oracle:
    """CPU restatement of ORAC's force path for one System."""

    def __init__(self, s, nthreads=None, ewald=True):
        self.s = s
        self.nthreads = nthreads or default_threads()
        self.ewald = ewald
        self.L = lib()
        self.lists = {}
        self.variant = None
        self.last_extra = np.zeros(4)
        self._prep()

    # -------------------------------------------------------- variants
    def set_rem(self, rematom, kind=0, factor=1.0):
        """force_rem (src/force_REM.f) for every later shell call."""
        self._rem = np.ascontiguousarray(rematom, dtype=np.uint8)
        v = Variant()
        v.mode = 1
        v.rematom = self._rem.ctypes.data
        v.rem_kind = int(kind)
        v.rem_factor = float(factor)
        self.variant = v

    def set_alchemy(self, ss_alchemy, qsoft=0.5, ljsoft=0.5, opls=False, shifted=False, qshift=0.0, ljshift=0.0):
        """force_alchemy (src/force_alchemy.f) with ORAC's per-atom soft-core
        parameters (src/mtsmd.f:1298-1303), or with `shifted` the
        shifted potential of force_ALCHEMY_shift (src/force_alchemy_shifted.f,
        ORAC's SHIFT-POT qshift ljshift); lambdas start at 0 (all on)."""
        rmin, epsm = self.s.alchemy_params()
        self._alch = (_i(ss_alchemy), _f(rmin), _f(epsm))
        v = Variant()
        v.mode = 2
        v.ss_alchemy = self._alch[0].ctypes.data
        v.rmin = self._alch[1].ctypes.data
        v.epsm = self._alch[2].ctypes.data
        v.qsoft = float(qsoft)
        v.ljsoft = float(ljsoft)
        v.opls = int(opls)
        v.shifted = int(bool(shifted))
        v.qshift = float(qshift)
        v.ljshift = float(ljshift)
        self.variant = v
        self.set_lambda(0.0, 0.0, 0.0, 0.0)

    def set_lambda(self, ladd, lrm, laddq, lrmq, ladd0=None, lrm0=None, laddq0=None, lrmq0=None, intramol=False,
                   ljintra=False):
        """Current and previous lambdas (cpropar ladd..lrmq0); the previous
        ones default to the current (zero work)."""
        v = self.variant
        ladd0 = ladd if ladd0 is None else ladd0
        lrm0 = lrm if lrm0 is None else lrm0
        laddq0 = laddq if laddq0 is None else laddq0
        lrmq0 = lrmq if lrmq0 is None else lrmq0
        v.fact[:] = alch_set(ladd, lrm, intramol, ljintra, False).ravel()
        v.factq[:] = alch_set(laddq, lrmq, intramol, ljintra, True).ravel()
        v.fact0[:] = alch_set(ladd0, lrm0, intramol, ljintra, False).ravel()
        v.factq0[:] = alch_set(laddq0, lrmq0, intramol, ljintra, True).ravel()

    def clear_variant(self):
        self.variant = None

    # ---------------------------------------------------------- bonded
    def intra_n0(self):
        """The bonded terms of mts_intra_n0 (src/mts_intra_n0.f:73-100):
        fpbond + fpbend + fitors.  Returns (F (3,N), {name: (slt, slv)})."""
        s = self.s
        r = self.cartesian()
        x, y, z = _f(r[0]), _f(r[1]), _f(r[2])
        fx, fy, fz = np.zeros(s.ntap), np.zeros(s.ntap), np.zeros(s.ntap)
        e = {}
        ss = _i(s.ss_index)
        ue = np.zeros(2)
        if s.bond_k is not None and len(s.bonds):
            self.L.orc_fpbond(ss, _i(s.bonds.ravel()), len(s.bonds), x, y, z, _f(s.bond_r0), _f(s.bond_k), ue, fx,
                              fy, fz)
        e["bond"] = tuple(ue)
        ue = np.zeros(2)
        if s.bends is not None and len(s.bends):
            self.L.orc_fpbend(ss, _i(s.bends.ravel()), len(s.bends), x, y, z, _f(s.bend_pot().ravel()), ue, fx, fy, fz)
        e["bend"] = tuple(ue)
        ue = np.zeros(2)
        self.last_skipped = 0
        if s.itors is not None and len(s.itors):
            self.last_skipped = self.L.orc_fitors(ss, _i(s.itors.ravel()), len(s.itors), x, y, z, _f(s.itors_a),
                                                  _f(s.itors_b), _f(s.itors_c), ue, fx, fy, fz)
        e["itors"] = tuple(ue)
        return np.stack([fx, fy, fz]), e

    def intra_torsions(self):
        """fptors (src/fptors.f), the torsion part of mts_intra_n1."""
        s = self.s
        r = self.cartesian()
        fx, fy, fz = np.zeros(s.ntap), np.zeros(s.ntap), np.zeros(s.ntap)
        ue = np.zeros(2)
        self.last_skipped = 0
        if s.tors is not None and len(s.tors):
            self.last_skipped = self.L.orc_fptors(_i(s.ss_index), _i(s.tors.ravel()), len(s.tors), _f(r[0]),
                                                  _f(r[1]), _f(r[2]), _f(s.tors_n), _f(s.tors_k), ue, fx, fy, fz)
        return np.stack([fx, fy, fz]), tuple(ue)

    def _prep(self):
        s = self.s
        self.co = _colmajor(s.co)
        self.oc = _colmajor(s.oc)
        self.type_cm = _i(np.asarray(s.type_table).T.ravel())
        self.grppt = _i(s.grppt.ravel())
        self.xp0, self.yp0, self.zp0 = _f(s.xp0), _f(s.yp0), _f(s.zp0)
        xg, yg, zg = s.group_centres()
        self.xpg, self.ypg, self.zpg = _f(xg), _f(yg), _f(zg)
        xm, ym, zm = s.molecule_centres()
        self.xpcm, self.ypcm, self.zpcm = _f(xm), _f(ym), _f(zm)

    def set_coords(self, xp0, yp0, zp0):
        self.s.xp0, self.s.yp0, self.s.zp0 = _f(xp0), _f(yp0), _f(zp0)
        self._prep()

    # ------------------------------------------------------------ lists
    def lc_list(self, rcut):
        s = self.s
        ncx, ncy, ncz = s.ncell
        indmax = (2 * ncx) * (2 * ncy) * (2 * ncz) + 1
        ii = np.zeros(indmax, np.int32)
        jj = np.zeros(indmax, np.int32)
        kk = np.zeros(indmax, np.int32)
        nind = self.L.orc_lc_index(indmax, ncx, ncy, ncz, rcut, self.co, ii, jj, kk)
        if nind < 0:
            raise RuntimeError(f"lc_index failed ({nind})")
        cap = s.ngrp * (s.ngrp + 1) // 2 + s.ngrp + 16
        cap = min(cap, 400_000_000)
        out = np.zeros(cap, np.int32)
        n = self.L.orc_lc_list(ncx, ncy, ncz, nind, ii, jj, kk, rcut, self.co, self.xpg, self.ypg, self.zpg, s.ngrp,
                               out, cap)
        if n < 0:
            raise RuntimeError("lc_list overflow")
        return out[:n].copy()

    def full_list(self):
        """ORAC's 'u' list for the brute-force update (iz = 0): one shared
        list [ngrp, 1..ngrp] read from mbeg = i+1."""
        return np.concatenate([[self.s.ngrp], np.arange(1, self.s.ngrp + 1)]).astype(np.int32)

    # ------------------------------------------------------------ force
    def force(self, nnlpp, rneigh, rinn, rout, rtolinn, rtolout, iz=1, lskip=None):
        """One call of force (src/force.f).  Returns (F (3,N), ue[6], stress
        (3,3), next list or None)."""
        s = self.s
        if lskip is None:
            lskip = bool(self.L.orc_decide_force(rinn, s.alphal)) if self.ewald else True
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        ue = np.zeros(6)
        st = np.zeros(9)
        nnlpp = _i(nnlpp)
        cap1 = len(nnlpp) + s.ngrp + 16
        if iz == 0:  # one shared list read from i+1: up to ngrp(ngrp-1)/2 pairs
            cap1 = s.ngrp * (s.ngrp + 1) // 2 + s.ngrp + 16
        nxt = np.zeros(cap1, np.int32)
        extra = np.zeros(4)
        n1 = self.L.orc_force_ex(_i(s.ss_index), self.xp0, self.yp0, self.zp0, self.xpg, self.ypg, self.zpg,
                                 _f(s.charge), _i(s.nbtype), self.type_cm, s.ntype, s.ntap, _i(s.atomg), self.xpcm,
                                 self.ypcm, self.zpcm, _i(s.atomp), self.co, _f(s.ecc12), _f(s.ecc6), s.alphal,
                                 _i(s.mapnl), s.ngrp, self.grppt, ue, fx, fy, fz, st, nnlpp, nxt, cap1, rneigh, rinn,
                                 rout, rtolinn, rtolout, _f(s.pmass), iz, _f(s.mass), s.massinfty, int(lskip),
                                 int(self.ewald), self.nthreads,
                                 C.byref(self.variant) if self.variant is not None else None, extra)
        self.last_extra = extra
        if n1 < 0:
            raise RuntimeError("next list overflow")
        nxt = nxt[:n1].copy() if rinn > 1e-5 else None
        return np.stack([fx, fy, fz]), ue, st.reshape(3, 3, order="F"), nxt

    def shell_params(self, shell, sh=None):
        """mts_forces radius selection, src/mts_forces.f:57-93:
        returns (ro, ri, rto, rti, rni, iz)."""
        sh = sh or self.s.shells
        if shell == "h":
            return sh.rcuth, sh.rcutl, sh.rtolh, sh.rtoll, sh.rneil, (1 if sh.rneih >= 1e-10 else 0)
        if shell == "l":
            return sh.rcutl, sh.rcutm, sh.rtoll, sh.rtolm, sh.rneim, 1
        if shell == "m":
            return sh.rcutm, 0.0, sh.rtolm, 0.0, 0.0, 1
        raise ValueError(shell)

    def mts_forces(self, shell, nnlpp, sh=None):
        ro, ri, rto, rti, rni, iz = self.shell_params(shell, sh)
        return self.force(nnlpp, rni, ri, ro, rti, rto, iz=iz)

    def update_lists(self):
        """Linked-cell H list plus the two phony calls that derive the L and
        M lists (src/mtsmd.f:2403-2470)."""
        import dataclasses

        sh = self.s.shells
        if self.s.ncell is None:
            # no LINKED_CELL: the 'u' shell over the all-pairs list (iz = 0),
            # src/mtsmd.f:2409-2418 with src/mts_forces.f:57-65
            _, _, _, self.lists["h"] = self.force(self.full_list(), sh.rneih, sh.rcuth, sh.rcuth, sh.rtolh, 0.0,
                                                  iz=0)
        else:
            self.lists["h"] = self.lc_list(sh.rcuth + sh.rtolh + sh.rneih)
        sh1 = dataclasses.replace(sh, rcuth=sh.rcutl, rtolh=0.0)
        _, _, _, self.lists["l"] = self.mts_forces("h", self.lists["h"], sh1)
        sh2 = dataclasses.replace(sh1, rcutl=sh.rcutm, rtoll=0.0)
        _, _, _, self.lists["m"] = self.mts_forces("l", self.lists["l"], sh2)

    def shell(self, shell):
        """Evaluate one shell with the current lists; H and L calls refresh
        the next inner list as ORAC's do."""
        F, ue, st, nxt = self.mts_forces(shell, self.lists[shell])
        if shell == "h":
            self.lists["l"] = nxt
        elif shell == "l":
            self.lists["m"] = nxt
        return F, ue, st

    def refresh_m_list(self):
        """Phony 'l' call after the H shell (src/mtsmd.f:3287-3295)."""
        import dataclasses

        sh = self.s.shells
        sh2 = dataclasses.replace(sh, rcutl=sh.rcutm)
        _, _, _, self.lists["m"] = self.mts_forces("l", self.lists["l"], sh2)

    # -------------------------------------------------------------- PME
    def fft_pme(self, pressure=True):
        s = self.s
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        eer = np.zeros(1)
        st = np.zeros(9)
        n1, n2, n3 = s.nfft
        self.L.orc_fft_pme(s.ntap, self.xp0, self.yp0, self.zp0, self.xpcm, self.ypcm, self.zpcm, _f(s.charge),
                           self.co, self.oc, s.volume, s.alphal, s.order, n1, n2, n3, eer, fx, fy, fz, st,
                           _i(s.atomp), int(pressure), s.rkcut, self.nthreads)
        return np.stack([fx, fy, fz]), float(eer[0]), st.reshape(3, 3, order="F")

    def do_pmesh_kspace(self, x, y, z, charge, recip, volume, alpha, order, nfft, rkcut=1e9):
        n = len(x)
        dx = np.zeros(n)
        dy = np.zeros(n)
        dz = np.zeros(n)
        eer = np.zeros(1)
        vir = np.zeros(9)
        self.L.orc_do_pmesh_kspace(n, _f(x), _f(y), _f(z), _f(charge), _colmajor(recip), volume, alpha, order,
                                   nfft[0], nfft[1], nfft[2], eer, dx, dy, dz, vir, rkcut, self.nthreads)
        return np.stack([dx, dy, dz]), float(eer[0]), vir.reshape(3, 3, order="F")

    # ------------------------------------------------------ corrections
    def cartesian(self):
        return self.s.cartesian()

    def ferrf(self, pairs, fudge, iz=1):
        s = self.s
        r = self.cartesian()
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        fs = np.zeros(2)
        p = _i(np.asarray(pairs).reshape(-1, 2).ravel())
        self.L.orc_ferrf(_i(s.ss_index), s.alphal, _f(s.charge), fudge, _f(r[0]), _f(r[1]), _f(r[2]), iz, p,
                         len(p) // 2, fs, fx, fy, fz)
        return np.stack([fx, fy, fz]), fs

    def cself(self):
        s = self.s
        a = np.zeros(1)
        b = np.zeros(1)
        self.L.orc_cself(_i(s.ss_index), _f(s.charge), s.ntap, s.alphal, s.rkcut, a, b)
        return float(a[0]), float(b[0])

    def fnb14(self, cut=True):
        s = self.s
        r = self.cartesian()
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        ue = np.zeros(4)
        p = _i(s.int14.ravel())
        self.L.orc_fnb14(_i(s.ss_index), _f(r[0]), _f(r[1]), _f(r[2]), _f(s.charge), s.ntap, _f(s.ecc1412),
                         _f(s.ecc146), int(cut), int(self.ewald), s.alphal, p, len(p) // 2, _i(s.type14), s.fudge,
                         1.0, fx, fy, fz, ue)
        return np.stack([fx, fy, fz]), ue

    def fnbgrp(self):
        s = self.s
        r = self.cartesian()
        fx = np.zeros(s.ntap)
        fy = np.zeros(s.ntap)
        fz = np.zeros(s.ntap)
        ue = np.zeros(4)
        p = _i(s.ingrp.ravel())
        self.L.orc_fnbgrp(_i(s.ss_index), _f(r[0]), _f(r[1]), _f(r[2]), _f(s.charge), _i(s.nbtype), _f(s.ecc12),
                          _f(s.ecc6), int(self.ewald), s.alphal, p, len(p) // 2, fx, fy, fz, ue)
        return np.stack([fx, fy, fz]), ue


    # ------------------------------------------- intra-alchemical terms
    def alch_lambdas(self, ss_alchemy, ladd, lrm):
        """Per-atom lambdas of the species (added ladd, removed -lrm)."""
        lam = np.zeros(self.s.ntap)
        self.L.orc_alch_atom_lambdas(self.s.ntap, _i(ss_alchemy), float(ladd), float(lrm), lam)
        return lam

    def alch_listqq(self, ss_alchemy):
        """listqq (src/initialize_lambda.f:62-139): (ia, ib, facQ) 1-based
        for the pairs of alchemical atoms beyond 1-4."""
        s = self.s
        excl = [np.asarray(a).reshape(-1, 2) for a in (s.bonds, s.constraints, s.bend13, s.int14) if len(a)]
        ex = _i(np.concatenate(excl).ravel()) if excl else _i(np.zeros(0))
        nal = int(np.sum(np.abs(np.asarray(ss_alchemy)) == 2))
        cap = max(1, nal * (nal - 1) // 2)
        out = np.zeros(3 * cap, np.int32)
        n = self.L.orc_alch_listqq(s.ntap, _i(ss_alchemy), ex, len(ex) // 2, out, cap)
        return out[:3 * n].reshape(-1, 3)

    def ferrf_alchemy_add(self, listqq, lamq, lamq0=None, intramol=False):
        """ferrf_alchemy_add (src/ferrf_alchemy_add.f) with the full charges:
        (F, (E slt, E slv), U(lambda) - U(lambda0))."""
        s = self.s
        r = self.cartesian()
        f = [np.zeros(s.ntap) for _ in range(3)]
        fs = np.zeros(2)
        dw = np.zeros(1)
        lq0 = lamq if lamq0 is None else lamq0
        lst = _i(np.asarray(listqq).ravel())
        self.L.orc_ferrf_alchemy_add(_i(s.ss_index), s.alphal, _f(s.charge), _f(lamq), _f(lq0), _f(r[0]), _f(r[1]),
                                     _f(r[2]), lst, len(lst) // 3, int(intramol), fs, dw, *f)
        return np.stack(f), fs, float(dw[0])

    def fnb14_alchemy(self, lam, lamq, lam0=None, lamq0=None):
        """fnb14_alchemy's Ewald branch (src/fnb14_alchemy.f:225-341) with
        the full charges: (F, (LJ slt, slv, Coulomb slt, slv), work)."""
        s = self.s
        r = self.cartesian()
        f = [np.zeros(s.ntap) for _ in range(3)]
        ue = np.zeros(4)
        dw = np.zeros(1)
        l0 = lam if lam0 is None else lam0
        lq0 = lamq if lamq0 is None else lamq0
        p = _i(s.int14.ravel())
        self.L.orc_fnb14_alchemy(_i(s.ss_index), _f(r[0]), _f(r[1]), _f(r[2]), _f(s.charge), _f(s.ecc1412),
                                 _f(s.ecc146), s.alphal, p, len(p) // 2, _i(s.type14), s.fudge, 1.0, _f(lam),
                                 _f(lamq), _f(l0), _f(lq0), *f, ue, dw)
        return np.stack(f), ue, float(dw[0])


class OracleMD:
    """CPU restatement of ORAC's NVE r-RESPA loop (orac_md.c)."""

    REC = 16  # doubles per energy record (orac_oracle.h)

    def __init__(self, s, dt_h, lrespa, mrespa, nupdte, rshk="l", nthreads=None, econst=0.0, n1respa=1, n0respa=1):
        L = lib()
        self.L = L
        self.s = s
        vp = C.c_void_p
        L.orc_md_create.restype = vp
        L.orc_md_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _I, _I, _I, _I, _I, _D, _D, _D, _D,
                                    _D, C.c_double, _D, _D, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_double, _D, C.c_int, C.c_int, C.c_int, _I, _D, C.c_int, C.c_double, C.c_int,
                                    C.c_int, C.c_int, C.c_char, _D, _D, C.c_int, C.c_double]
        L.orc_md_run.restype = C.c_int
        L.orc_md_run.argtypes = [vp, C.c_int, C.c_int, _D]
        L.orc_md_get_state.argtypes = [vp, _D, _D]
        L.orc_md_destroy.argtypes = [vp]
        sh = s.shells
        self._keep = dict(
            ss=_i(s.ss_index), nbt=_i(s.nbtype), tt=_i(np.asarray(s.type_table).T.ravel()), ag=_i(s.atomg),
            ap=_i(s.atomp), gp=_i(s.grppt.ravel()), mp=_i(s.mapnl), q=_f(s.charge), e12=_f(s.ecc12), e6=_f(s.ecc6),
            m=_f(s.mass), pm=_f(s.pmass), co=_colmajor(s.co), oc=_colmajor(s.oc),
            sh=_f([sh.rcutm, sh.rtolm, sh.rneim, sh.rcutl, sh.rtoll, sh.rneil, sh.rcuth, sh.rtolh, sh.rneih]),
            cn=_i(s.constraints.ravel()), dss=_f(s.cdist ** 2))
        k = self._keep
        x = _f(s.cartesian().ravel())
        v = _f(np.concatenate([s.vx, s.vy, s.vz]))
        n1, n2, n3 = s.nfft
        self.h = L.orc_md_create(s.ntap, s.ngrp, s.nprot, s.ntype, k["ss"], k["nbt"], k["tt"], k["ag"], k["ap"],
                                 k["gp"], k["mp"], k["q"], k["e12"], k["e6"], k["m"], k["pm"], s.massinfty, k["co"],
                                 k["oc"], s.alphal, s.order, n1, n2, n3, s.rkcut, k["sh"], *s.ncell, k["cn"],
                                 k["dss"], len(s.constraints), dt_h, lrespa, mrespa, nupdte, rshk.encode(), x, v,
                                 nthreads or default_threads(), econst)
        if not self.h:
            raise RuntimeError("orc_md_create failed")
        a = intra_lists(s)
        if n1respa != 1 or n0respa != 1 or any(len(a[k]) for k in ("lbnd", "lbndg", "ltor", "litr", "int14", "ingrp",
                                                                     "int13")):
            L.orc_md_set_intra.argtypes = [vp, C.c_int, _I, _D, _D, C.c_int, _I, _D, C.c_int, _I, _D, _D, C.c_int,
                                           _I, _D, _D, _D, C.c_int, _I, _I, _D, _D, C.c_int, C.c_double, C.c_int,
                                           _I, C.c_int, _I, C.c_int, C.c_int]
            self._keep["intra"] = a
            L.orc_md_set_intra(self.h, len(a["lbnd"]) // 2, a["lbnd"], a["r0"], a["kb"], len(a["lbndg"]) // 3,
                               a["lbndg"], a["bendpot"], len(a["ltor"]) // 4, a["ltor"], a["tpota"], a["tpotb"],
                               len(a["litr"]) // 4, a["litr"], a["ipota"], a["ipotb"], a["ipotc"],
                               len(a["int14"]) // 2, a["int14"], a["type14"], a["ecc1412"], a["ecc146"],
                               len(a["ecc1412"]), s.fudge, len(a["ingrp"]) // 2, a["ingrp"], len(a["int13"]) // 2,
                               a["int13"], n1respa, n0respa)

    def set_alchemy(self, ss_alchemy, lam8, qsoft=0.5, ljsoft=0.5, opls=False, shifted=False, qshift=0.0,
                    ljshift=0.0, intramol=False, ljintra=False):
        """Alchemy in the loop (force_alchemy, do_pmesh_alchemy, ferrf over
        the scaled charges, fnb14_alchemy, ferrf_alchemy_add over listqq):
        lam8 = ladd lrm laddq lrmq ladd0 lrm0 laddq0 lrmq0."""
        L, s = self.L, self.s
        vp = C.c_void_p
        rmin, epsm = s.alchemy_params()
        lq = Oracle(s, nthreads=1).alch_listqq(ss_alchemy)
        self._keep["alch"] = (_i(ss_alchemy), _f(rmin), _f(epsm), _f(lam8), _i(lq.ravel()))
        a = self._keep["alch"]
        L.orc_md_set_alchemy.argtypes = [vp, _I, _D, _D, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                         C.c_double, C.c_int, C.c_int, _D, _I, C.c_int]
        L.orc_md_set_alchemy(self.h, a[0], a[1], a[2], qsoft, ljsoft, int(opls), int(bool(shifted)), qshift,
                             ljshift, int(intramol), int(ljintra), a[3], a[4], len(lq))

    def set_schedule(self, times_fs, ladded, laddedq, lremoved, lremovedq, t0=0.0):
        """A non-equilibrium run (alchemic): the lambdas follow the schedule
        from t0 (fs) on, the work starts at 0."""
        L = self.L
        sch = [_f(times_fs), _f(ladded), _f(laddedq), _f(lremoved), _f(lremovedq)]
        self._keep["schedule"] = sch
        L.orc_md_set_schedule.argtypes = [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, C.c_double]
        L.orc_md_set_schedule(self.h, len(sch[0]), *sch, float(t0))

    def set_thermostat(self, temp, nu_com, nu_solute, nu_solvent):
        """ORAC's THERMOS: Nose-Hoover thermostats of the molecular centres
        of mass, the solute and the solvent at temp (K), frequencies in cm^-1."""
        self.L.orc_md_set_thermostat.argtypes = [C.c_void_p, C.c_double, _D]
        self.L.orc_md_set_thermostat(self.h, float(temp), _f([nu_com, nu_solute, nu_solvent]))

    def set_thermostat_state(self, eta, etap):
        """A restart's thermostat coordinates and velocities."""
        self.L.orc_md_set_thermostat_state.argtypes = [C.c_void_p, _D, _D]
        self.L.orc_md_set_thermostat_state(self.h, _f(eta), _f(etap))

    def thermostat(self):
        """(eta[3], etap[3], Q[3], ndf[3], energy) of the three thermostats."""
        out = np.zeros(13)
        self.L.orc_md_thermostat.argtypes = [C.c_void_p, _D]
        self.L.orc_md_thermostat(self.h, out)
        return out[0:3].copy(), out[3:6].copy(), out[6:9].copy(), out[9:12].astype(int), float(out[12])

    def work(self):
        """(work, rtime, (ladd, lrm, laddq, lrmq), latest work terms[8])."""
        out = np.zeros(14)
        self.L.orc_md_work.argtypes = [C.c_void_p, _D]
        self.L.orc_md_work(self.h, out)
        return float(out[0]), float(out[1]), tuple(out[2:6]), out[6:14].copy()

    def run(self, nsteps, energy_every=0):
        R = self.REC
        nrec = nsteps // energy_every if energy_every else 0
        rec = np.zeros(max(1, nrec) * R)
        rc = self.L.orc_md_run(self.h, nsteps, energy_every, rec)
        if rc:
            raise RuntimeError(f"orc_md_run status {rc}")
        return rec[:nrec * R].reshape(-1, R)

    def state(self):
        n = self.s.ntap
        x = np.zeros(3 * n)
        v = np.zeros(3 * n)
        self.L.orc_md_get_state(self.h, x, v)
        return x.reshape(3, n), v.reshape(3, n)

    def close(self):
        if self.h:
            self.L.orc_md_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rel_rms(F, Fref):
    """ORAC's check_force metric (src/pme_code.f:378-396)."""
    return float(np.sqrt(((F - Fref) ** 2).sum() / (Fref ** 2).sum()))
