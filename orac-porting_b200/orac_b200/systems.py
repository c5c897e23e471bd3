"""Synthetic ORAC systems in ORAC's own array conventions.

Every array follows the Fortran layout that ORAC's force path reads from its
module globals (src/mts_forces.f:120-152): 1-based indices stored in int32
arrays, coordinates in scaled box units s in [-1, 1) with r = co s
(src/setuns.f:43, src/force.f:268-276), charges and LJ tables in internal
units (src/covchg.f:37-39, src/covnb.f).

Builders:
  water_box(...)      3-site rigid TIP3P-like water box (the 3,000-water
                      31 A workload and its liquid-density variant)
  polymer_in_water()  bonded chain + water (22,700-atom workload)
  two_groups(...)     hand-checkable small cases
"""
from __future__ import annotations

import dataclasses
import math
from collections import defaultdict

import numpy as np

from . import units


@dataclasses.dataclass
class Shells:
    """r-RESPA shell radii (MTS_RESPA `step nonbond n rcut rtol rnei`,
    src/read_integrator.f:152-230, defaults :491-527)."""

    rcutm: float = 5.0
    rtolm: float = 0.3
    rneim: float = 0.4
    rcutl: float = 7.5
    rtoll: float = 0.3
    rneil: float = 0.5
    rcuth: float = 10.0
    rtolh: float = 0.3
    rneih: float = 1.5


@dataclasses.dataclass
class System:
    name: str
    ntap: int
    ngrp: int
    nprot: int
    co: np.ndarray  # (3,3) float64, co[i,j] = co(i+1,j+1)
    xp0: np.ndarray  # scaled coordinates
    yp0: np.ndarray
    zp0: np.ndarray
    mass: np.ndarray
    charge: np.ndarray  # internal units
    nbtype: np.ndarray  # int32, 1-based LJ type
    ntype: int
    type_table: np.ndarray  # (ntype, ntype) int32, 1-based index into ecc tables
    ecc12: np.ndarray
    ecc6: np.ndarray
    grppt: np.ndarray  # (ngrp, 2) int32 1-based first/last atom
    atomg: np.ndarray  # int32 1-based group of each atom
    atomp: np.ndarray  # int32 1-based molecule of each atom
    ss_index: np.ndarray  # int32: 1 solute, 2 solvent
    pmass: np.ndarray  # mass fraction of each atom within its group
    mapnl: np.ndarray  # int32 serial exclusion map [n, j1..jn] per atom
    int14: np.ndarray  # (n14, 2) int32 1-based
    type14: np.ndarray  # (n14,) int32 1-based into ecc1412/ecc146
    ecc1412: np.ndarray
    ecc146: np.ndarray
    ingrp: np.ndarray  # (ningrp, 2) non-excluded pairs inside one group
    bonds: np.ndarray  # (nb, 2) flexible bonds (ferrf list lstrtch)
    bend13: np.ndarray  # (n13, 2) 1-3 pairs (ferrf list int13)
    constraints: np.ndarray  # (nc, 2) rigid bonds
    cdist: np.ndarray  # (nc,) constraint lengths
    vx: np.ndarray  # Cartesian velocities, A/fs
    vy: np.ndarray
    vz: np.ndarray
    alphal: float = 0.35
    order: int = 4
    nfft: tuple = (32, 32, 32)
    shells: Shells = dataclasses.field(default_factory=Shells)
    fudge: float = 0.83333
    lj_fudge: float = 0.5
    ncell: tuple = (10, 10, 10)
    massinfty: float = 1.0e20
    rkcut: float = 1.0e9
    # bonded terms for flexible solutes (harmonic bonds / bends, cosine torsions)
    bond_k: np.ndarray | None = None
    bond_r0: np.ndarray | None = None
    bends: np.ndarray | None = None  # (na, 3)
    bend_k: np.ndarray | None = None
    bend_t0: np.ndarray | None = None
    bend_ub_r0: np.ndarray | None = None  # Urey-Bradley 1-3 spring (fpbend potc, potd)
    bend_ub_k: np.ndarray | None = None
    tors: np.ndarray | None = None  # (nt, 4)
    tors_k: np.ndarray | None = None  # fptors potb (V)
    tors_n: np.ndarray | None = None  # fptors pota: +-n, the sign selecting phase 0 or pi
    # improper torsions (fitors): atoms, pota, potb, potc (potc > 0: harmonic)
    itors: np.ndarray | None = None
    itors_a: np.ndarray | None = None
    itors_b: np.ndarray | None = None
    itors_c: np.ndarray | None = None
    lj_params: np.ndarray | None = None  # (ntype, 2): Rmin/2 (A), eps (kcal/mol) per LJ type
    # alchemy (soft-core force_alchemy): 1 normal, 2 added, -2 removed per atom
    ss_alchemy: np.ndarray | None = None
    # REM segment (force_rem): 1 for atoms of the scaled segment
    rematom: np.ndarray | None = None
    # Cartesian positions (3, N) saved when a resident system leaves the
    # device; the next md_setup starts from them exactly (xp0..zp0 hold the
    # same positions scaled, rounded)
    xyz_restart: np.ndarray | None = None

    def bend_pot(self):
        """fpbend's pota..potg per bend: theta0, k, Urey-Bradley r0 and k,
        no stretch-stretch coupling."""
        n = 0 if self.bends is None else len(self.bends)
        p = np.zeros((n, 7))
        if n:
            p[:, 0] = self.bend_t0
            p[:, 1] = self.bend_k
            if self.bend_ub_k is not None:
                p[:, 2] = self.bend_ub_r0
                p[:, 3] = self.bend_ub_k
        return p

    def intra_lists(self):
        """Flat 1-based lists and parameter arrays of the intramolecular
        terms: bonds (lbnd, r0, kb), bends (lbndg, bendpot), torsions (ltor,
        tpota, tpotb), impropers (litr, ipota..ipotc), 1-4 pairs (int14,
        type14, ecc1412, ecc146), intra-group pairs (ingrp), 1-3 pairs
        (int13)."""
        def ints(a, w):
            return np.ascontiguousarray(np.zeros((0, w)) if a is None else np.asarray(a).reshape(-1, w),
                                        dtype=np.int32).ravel()

        def dbl(a, n):
            return np.ascontiguousarray(np.zeros(n) if a is None else a, dtype=np.float64)

        has_b = self.bond_k is not None
        out = dict(lbnd=ints(self.bonds if has_b else None, 2))
        nb = len(out["lbnd"]) // 2
        out["r0"], out["kb"] = dbl(self.bond_r0 if has_b else None, nb), dbl(self.bond_k if has_b else None, nb)
        out["lbndg"] = ints(self.bends, 3)
        out["bendpot"] = dbl(self.bend_pot().ravel(), 0)
        out["ltor"] = ints(self.tors, 4)
        nt = len(out["ltor"]) // 4
        out["tpota"], out["tpotb"] = dbl(self.tors_n, nt), dbl(self.tors_k, nt)
        out["litr"] = ints(self.itors, 4)
        ni = len(out["litr"]) // 4
        out["ipota"], out["ipotb"], out["ipotc"] = dbl(self.itors_a, ni), dbl(self.itors_b, ni), dbl(self.itors_c, ni)
        out["int14"] = ints(self.int14, 2)
        out["type14"] = np.ascontiguousarray(self.type14 if len(self.int14) else np.zeros(0), dtype=np.int32)
        out["ecc1412"], out["ecc146"] = dbl(self.ecc1412, 0), dbl(self.ecc146, 0)
        out["ingrp"] = ints(self.ingrp, 2)
        out["int13"] = ints(self.bend13, 2)
        return out

    def has_intra(self):
        a = self.intra_lists()
        return any(len(a[k]) for k in ("lbnd", "lbndg", "ltor", "litr", "int14", "ingrp", "int13"))

    def alchemy_params(self):
        """Per-atom rmin, epsm of the soft-core kernel (src/mtsmd.f:1298-1303)."""
        p = self.lj_params[self.nbtype - 1]
        return units.alchemy_rmin_epsm(p[:, 0], p[:, 1])

    @property
    def oc(self):
        return np.linalg.inv(self.co)

    @property
    def volume(self):
        return 8.0 * abs(np.linalg.det(self.co))

    def cartesian(self):
        s = np.stack([self.xp0, self.yp0, self.zp0])
        return self.co @ s

    def group_centres(self):
        """appbou (src/appbou.f:57-69) in scaled coordinates."""
        g = self.atomg - 1
        out = []
        for c in (self.xp0, self.yp0, self.zp0):
            out.append(np.bincount(g, weights=self.pmass * c, minlength=self.ngrp))
        return out

    def molecule_centres(self):
        """Mass-weighted molecule centres in scaled coordinates."""
        p = self.atomp - 1
        mt = np.bincount(p, weights=self.mass, minlength=self.nprot)
        out = []
        for c in (self.xp0, self.yp0, self.zp0):
            out.append(np.bincount(p, weights=self.mass * c, minlength=self.nprot) / mt)
        return out

    def copy(self):
        return dataclasses.replace(
            self,
            **{
                f.name: (getattr(self, f.name).copy() if isinstance(getattr(self, f.name), np.ndarray) else getattr(self, f.name))
                for f in dataclasses.fields(self)
            },
        )


# ----------------------------------------------------------------- topology


def _exclusions(natoms_mol, bonds_mol):
    """1-2, 1-3, 1-4 partner sets of a molecule from its bond graph
    (the three sources mappa merges, src/mappa.f:60-125)."""
    adj = defaultdict(set)
    for a, b in bonds_mol:
        adj[a].add(b)
        adj[b].add(a)
    ex12 = {a: set(adj[a]) for a in range(natoms_mol)}
    ex13 = {a: set() for a in range(natoms_mol)}
    ex14 = {a: set() for a in range(natoms_mol)}
    for a in range(natoms_mol):
        for b in adj[a]:
            for c in adj[b]:
                if c != a:
                    ex13[a].add(c)
                    for d in adj[c]:
                        if d != b and d != a:
                            ex14[a].add(d)
    for a in range(natoms_mol):
        ex13[a] -= ex12[a]
        ex14[a] -= ex12[a] | ex13[a]
    return ex12, ex13, ex14


def _lj_tables(types):
    """types: list of (rmin_half, eps_kcal).  Returns type_table, ecc12, ecc6
    with ij = j*(j-1)/2 + i for i <= j (covnb.f)."""
    nt = len(types)
    npair = nt * (nt + 1) // 2
    e12 = np.zeros(npair)
    e6 = np.zeros(npair)
    tt = np.zeros((nt, nt), dtype=np.int32)
    for i in range(1, nt + 1):
        for j in range(i, nt + 1):
            ij = j * (j - 1) // 2 + i
            a, b = units.amber_pair(types[i - 1][0], types[i - 1][1], types[j - 1][0], types[j - 1][1])
            e12[ij - 1] = a
            e6[ij - 1] = b
            tt[i - 1, j - 1] = ij
            tt[j - 1, i - 1] = ij
    return tt, e12, e6


def _assemble(name, co, pos_cart, mass, q_e, ltype, lj_types, groups, molecules, bonds, solute_mask,
              constraints=(), seed_v=None, temperature=300.0, flexible_bonds=(), **kw):
    """Assemble a System from Cartesian positions and molecular topology.

    groups: list of (first, last) 0-based atom ranges, contiguous, ordered.
    molecules: list of (first, last) 0-based atom ranges.
    bonds: list of (a, b) 0-based (all bonds, rigid and flexible).
    """
    n = len(mass)
    co = np.asarray(co, dtype=np.float64)
    oc = np.linalg.inv(co)
    s = oc @ pos_cart
    grppt = np.array([[a + 1, b + 1] for a, b in groups], dtype=np.int32)
    atomg = np.zeros(n, dtype=np.int32)
    for g, (a, b) in enumerate(groups):
        atomg[a:b + 1] = g + 1
    atomp = np.zeros(n, dtype=np.int32)
    for m, (a, b) in enumerate(molecules):
        atomp[a:b + 1] = m + 1
    assert (atomg > 0).all() and (atomp > 0).all()
    gm = np.bincount(atomg - 1, weights=mass)
    pmass = mass / gm[atomg - 1]
    # exclusions per molecule
    bonds_by_mol = defaultdict(list)
    for a, b in bonds:
        assert atomp[a] == atomp[b]
        bonds_by_mol[atomp[a] - 1].append((a, b))
    excl = [set() for _ in range(n)]
    pairs14 = []
    pairs13 = []
    for m, (a0, a1) in enumerate(molecules):
        nm = a1 - a0 + 1
        bl = [(a - a0, b - a0) for a, b in bonds_by_mol.get(m, [])]
        if not bl:
            continue
        e12, e13, e14 = _exclusions(nm, bl)
        for a in range(nm):
            for b in e12[a] | e13[a] | e14[a]:
                if b > a:
                    excl[a0 + a].add(a0 + b)
            for b in e14[a]:
                if b > a:
                    pairs14.append((a0 + a, a0 + b))
            for b in e13[a]:
                if b > a:
                    pairs13.append((a0 + a, a0 + b))
    mapnl = []
    for a in range(n):
        js = sorted(excl[a])
        mapnl.append(len(js))
        mapnl.extend(j + 1 for j in js)
    mapnl = np.array(mapnl, dtype=np.int32)
    # non-excluded intra-group pairs (fnbgrp list)
    ingrp = []
    for a, b in groups:
        for i in range(a, b + 1):
            for j in range(i + 1, b + 1):
                if j not in excl[i]:
                    ingrp.append((i + 1, j + 1))
    tt, e12t, e6t = _lj_tables(lj_types)
    nt = len(lj_types)
    int14 = np.array([(a + 1, b + 1) for a, b in pairs14], dtype=np.int32).reshape(-1, 2)
    type14 = np.array([tt[ltype[a] - 1, ltype[b] - 1] for a, b in pairs14], dtype=np.int32)
    cset = set(tuple(sorted(c)) for c in constraints)
    flex = [tuple(sorted(b)) for b in bonds if tuple(sorted(b)) not in cset]
    cons = np.array([(a + 1, b + 1) for a, b in sorted(cset)], dtype=np.int32).reshape(-1, 2)
    cdist = np.array([np.linalg.norm(pos_cart[:, a] - pos_cart[:, b]) for a, b in sorted(cset)])
    rng = np.random.default_rng(seed_v if seed_v is not None else 4)
    # Maxwell-Boltzmann velocities, A/fs: sigma^2 = kT/m in internal units
    kT = units.BOLTZ * temperature / units.UNITE
    sig = np.sqrt(kT / mass)
    v = rng.standard_normal((3, n)) * sig
    ptot = (v * mass).sum(axis=1) / mass.sum()
    v -= ptot[:, None]
    ss = np.where(solute_mask, 1, 2).astype(np.int32)
    sysm = System(
        lj_params=np.array(lj_types, dtype=np.float64).reshape(-1, 2),
        name=name, ntap=n, ngrp=len(groups), nprot=len(molecules), co=co,
        xp0=s[0].copy(), yp0=s[1].copy(), zp0=s[2].copy(), mass=np.asarray(mass, dtype=np.float64),
        charge=np.array([units.charge_internal(q) for q in q_e]), nbtype=np.asarray(ltype, dtype=np.int32),
        ntype=nt, type_table=tt, ecc12=e12t, ecc6=e6t, grppt=grppt, atomg=atomg, atomp=atomp,
        ss_index=ss, pmass=pmass, mapnl=mapnl, int14=int14, type14=type14,
        ecc1412=e12t * kw.get("lj_fudge", 0.5), ecc146=e6t * kw.get("lj_fudge", 0.5),
        ingrp=np.array(ingrp, dtype=np.int32).reshape(-1, 2),
        bonds=np.array([(a + 1, b + 1) for a, b in flex], dtype=np.int32).reshape(-1, 2),
        bend13=np.array([(a + 1, b + 1) for a, b in pairs13], dtype=np.int32).reshape(-1, 2),
        constraints=cons, cdist=cdist, vx=v[0].copy(), vy=v[1].copy(), vz=v[2].copy(),
    )
    for k, val in kw.items():
        setattr(sysm, k, val)
    # ecc1412/ecc146 follow the fudge actually set
    sysm.ecc1412 = e12t * sysm.lj_fudge
    sysm.ecc146 = e6t * sysm.lj_fudge
    return sysm


# -------------------------------------------------------------------- water

R_OH = 0.957  # ff/amber99sb-ildn.prm:22-23 (TIP3P geometry)
R_HH = 1.514
Q_O, Q_H = -0.834, 0.417  # ff/amber99sb-ildn.tpg:3280-3282
M_O, M_H = 16.00, 1.008
SIGMA_O, EPS_O = 3.15, 0.152


def _water_template():
    half = math.asin(0.5 * R_HH / R_OH)
    h1 = np.array([R_OH * math.sin(half), R_OH * math.cos(half), 0.0])
    h2 = np.array([-R_OH * math.sin(half), R_OH * math.cos(half), 0.0])
    return np.stack([np.zeros(3), h1, h2])


def _random_rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
    ])


def water_lj_types():
    rmin_half_o = SIGMA_O * 2.0 ** (1.0 / 6.0) / 2.0
    return [(rmin_half_o, EPS_O), (0.0, 0.0)]


def water_box(nwat=3000, box=31.0, lattice=15, jitter=0.3, seeds=(1, 2, 3, 4), nfft=(32, 32, 32),
              alphal=0.35, order=4, ncell=None, name=None):
    """Cubic box of rigid 3-site waters on a jittered lattice.

    Defaults give the 3,000-water 31 A box: 15^3 lattice sites (spacing 31/15),
    3,000 kept by a seeded shuffle, O jitter U(+-0.3 A), random orientation,
    Maxwell-Boltzmann velocities at 300 K.  One group and one molecule per
    water; O-H, O-H, H-H are rigid bonds, all three intra pairs excluded.
    """
    r1, r2, r3, r4 = (np.random.default_rng(s) for s in seeds)
    nsite = lattice ** 3
    assert nwat <= nsite
    keep = np.sort(r1.permutation(nsite)[:nwat])
    a = box / lattice
    idx = np.stack(np.unravel_index(keep, (lattice,) * 3), axis=1).astype(np.float64)
    opos = (idx + 0.5) * a - 0.5 * box + r2.uniform(-jitter, jitter, size=(nwat, 3))
    tmpl = _water_template()
    pos = np.zeros((3, 3 * nwat))
    for w in range(nwat):
        R = _random_rotation(r3)
        for k in range(3):
            pos[:, 3 * w + k] = opos[w] + R @ tmpl[k]
    n = 3 * nwat
    mass = np.tile([M_O, M_H, M_H], nwat)
    q = np.tile([Q_O, Q_H, Q_H], nwat)
    lt = np.tile([1, 2, 2], nwat)
    groups = [(3 * w, 3 * w + 2) for w in range(nwat)]
    bonds = []
    cons = []
    for w in range(nwat):
        o = 3 * w
        for b in ((o, o + 1), (o, o + 2), (o + 1, o + 2)):
            bonds.append(b)
            cons.append(b)
    if ncell is None:
        ncell = (max(3, int(box / 3.1)),) * 3
    co = np.diag([box / 2.0] * 3)
    return _assemble(name or f"water{nwat}_L{box:g}", co, pos, mass, q, lt, water_lj_types(), groups, groups,
                     bonds, np.zeros(n, dtype=bool), constraints=cons, seed_v=seeds[3],
                     alphal=alphal, order=order, nfft=tuple(nfft), ncell=tuple(ncell))


def config1_water():
    """3,000 waters, 31.0 A cubic box, alpha 0.35, 32^3 grid order 4, shells
    0.5/2/4 fs at 5.0/7.5/10.0 A."""
    return water_box(name="config1_water3000")


def config1_liquid():
    """Same 3,000 waters at liquid density (44.7 A box, 48^3 grid)."""
    return water_box(box=44.7, nfft=(48, 48, 48), name="config1_liquid3000")


# ------------------------------------------------------------------ polymer


def _grow_chain(n, rng, bond=1.53, angle=112.0, box=None, center=None, clash=2.2, others=None, max_tries=100):
    """Self-avoiding chain growth with fixed bond length and angle and random
    torsions; a step that finds no free position backtracks a few atoms."""
    th = math.radians(angle)
    pos = [np.zeros(3) if center is None else np.array(center, dtype=float)]
    d0 = rng.standard_normal(3)
    d0 /= np.linalg.norm(d0)
    pos.append(pos[0] + bond * d0)
    stuck = 0
    while len(pos) < n:
        ok = False
        for _ in range(max_tries):
            b1 = pos[-1] - pos[-2]
            b1 /= np.linalg.norm(b1)
            if len(pos) >= 3:
                b0 = pos[-2] - pos[-3]
            else:
                b0 = rng.standard_normal(3)
            perp = b0 - np.dot(b0, b1) * b1
            perp /= np.linalg.norm(perp)
            phi = rng.uniform(-math.pi, math.pi)
            w = np.cross(b1, perp)
            dirn = -math.cos(th) * b1 + math.sin(th) * (math.cos(phi) * perp + math.sin(phi) * w)
            p = pos[-1] + bond * dirn
            arr = np.array(pos[:-3]) if len(pos) > 3 else np.zeros((0, 3))
            if len(arr):
                dd = arr - p
                if box is not None:
                    dd -= box * np.round(dd / box)
                if (np.einsum("ij,ij->i", dd, dd) < clash * clash).any():
                    continue
            ok = True
            break
        if not ok:
            stuck += 1
            if stuck > 1000 or len(pos) < 8:
                raise RuntimeError("chain growth failed")
            del pos[-5:]
            continue
        pos.append(p)
    return np.array(pos)


NTYPE_CHAIN = 64


def polymer_in_water(nchain=1700, nwat=7000, box=62.0, seed_chain=5, seed_lj=6, seed_wat=7, nfft=(64, 64, 64),
                     order=5, alphal=0.35, name="config2_polymer22700", group_size=3, ncell=None):
    """Bonded polymer chain in water (22,700 atoms in the default sizes).

    Chain: bond 1.53 A, angle 112 deg, random torsions, seeded self-avoiding
    growth; groups of 3 consecutive atoms; charges N(0, 0.35) neutralised per
    group then per chain; 64 chain LJ types with sigma U[2.0, 3.8] A and eps
    U[0.02, 0.2] kcal/mol, assigned to chain atoms at random;
    1-2/1-3 excluded, 1-4 scaled (LJ 0.5, QQ 0.8333).  Waters: the water_box
    molecule, inserted at random with overlap rejection at 2.4 A.
    """
    rng = np.random.default_rng(seed_chain)
    chain = _grow_chain(nchain, rng, box=box)
    chain -= chain.mean(axis=0)
    # wrap the chain as a whole molecule: keep it unwrapped (one molecule)
    rl = np.random.default_rng(seed_lj)
    q = rng.normal(0.0, 0.35, nchain)
    cgroups = [(a, min(a + group_size - 1, nchain - 1)) for a in range(0, nchain, group_size)]
    for a, b in cgroups:
        q[a:b + 1] -= q[a:b + 1].mean()
    q -= q.mean()
    # LJ types of the chain: NTYPE_CHAIN (sigma, eps) pairs drawn from the
    # stated ranges, one type assigned to each chain atom at random
    sig = rl.uniform(2.0, 3.8, NTYPE_CHAIN)
    eps = rl.uniform(0.02, 0.2, NTYPE_CHAIN)
    chain_types = [(s_ * 2.0 ** (1.0 / 6.0) / 2.0, e_) for s_, e_ in zip(sig, eps)]
    chain_lt = rl.integers(1, NTYPE_CHAIN + 1, nchain)
    # waters by rejection
    rw = np.random.default_rng(seed_wat)
    tmpl = _water_template()
    placed = []
    cell = 3.0
    nc = int(box // cell)
    grid = defaultdict(list)

    def cell_of(p):
        return tuple((np.floor((p + box / 2) / (box / nc)).astype(int)) % nc)

    def clashes(p):
        c = cell_of(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for qpos in grid.get(((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc), ()):
                        d = p - qpos
                        d -= box * np.round(d / box)
                        if d @ d < 2.4 * 2.4:
                            return True
        return False

    for p in chain:
        grid[cell_of(p)].append(p)
    tries = 0
    while len(placed) < nwat:
        tries += 1
        if tries > 200 * nwat:
            raise RuntimeError("water insertion failed")
        o = rw.uniform(-box / 2, box / 2, 3)
        if clashes(o):
            continue
        R = _random_rotation(rw)
        mol = np.stack([o + R @ t for t in tmpl])
        placed.append(mol)
        grid[cell_of(o)].append(o)
    n = nchain + 3 * nwat
    pos = np.zeros((3, n))
    pos[:, :nchain] = chain.T
    for w, mol in enumerate(placed):
        pos[:, nchain + 3 * w:nchain + 3 * w + 3] = mol.T
    mass = np.concatenate([np.full(nchain, 12.011), np.tile([M_O, M_H, M_H], nwat)])
    qa = np.concatenate([q, np.tile([Q_O, Q_H, Q_H], nwat)])
    types = chain_types + water_lj_types()
    lt = np.zeros(n, dtype=np.int32)
    lt[:nchain] = chain_lt
    lt[nchain:] = np.tile([NTYPE_CHAIN + 1, NTYPE_CHAIN + 2, NTYPE_CHAIN + 2], nwat)
    groups = cgroups + [(nchain + 3 * w, nchain + 3 * w + 2) for w in range(nwat)]
    molecules = [(0, nchain - 1)] + [(nchain + 3 * w, nchain + 3 * w + 2) for w in range(nwat)]
    bonds = [(i, i + 1) for i in range(nchain - 1)]
    cons = []
    for w in range(nwat):
        o = nchain + 3 * w
        for b in ((o, o + 1), (o, o + 2), (o + 1, o + 2)):
            bonds.append(b)
            cons.append(b)
    solute = np.zeros(n, dtype=bool)
    solute[:nchain] = True
    co = np.diag([box / 2.0] * 3)
    s = _assemble(name, co, pos, mass, qa, lt, types, groups, molecules, bonds, solute, constraints=cons,
                  seed_v=4, alphal=alphal, order=order, nfft=tuple(nfft),
                  ncell=ncell if ncell is not None else (int(box / 3.1),) * 3,
                  fudge=0.8333, lj_fudge=0.5)
    # bonded terms of the chain: harmonic bond 1.53 A, harmonic angle 112 deg,
    # 3-fold cosine torsion
    s.bond_k = np.full(len(s.bonds), 300.0 * 4184.0 / units.EFACT)
    s.bond_r0 = np.full(len(s.bonds), 1.53)
    s.bends = np.array([(i + 1, i + 2, i + 3) for i in range(nchain - 2)], dtype=np.int32)
    s.bend_k = np.full(len(s.bends), 60.0 * 4184.0 / units.EFACT)
    s.bend_t0 = np.full(len(s.bends), math.radians(112.0))
    s.tors = np.array([(i + 1, i + 2, i + 3, i + 4) for i in range(nchain - 3)], dtype=np.int32)
    s.tors_k = np.full(len(s.tors), 1.4 * 4184.0 / units.EFACT)
    s.tors_n = np.full(len(s.tors), -3.0)  # U = V cos(3 phi) - V: trans minimum
    return s


def ligand_in_water(nlig=40, seed=8, box=44.7, nwat=3000, nfft=(48, 48, 48), group_size=3, remove_within=2.4,
                    name="ligand40_liquid"):
    """A flexible 40-atom ligand (a chain fragment built like the polymer:
    bond 1.53 A, angle 112 deg, random torsions, charges N(0, 0.35)
    neutralised per group and per molecule, LJ types drawn from the chain
    types) at the centre of the liquid-density water box, with every water
    whose oxygen lies within 2.4 A of a ligand atom removed.  The ligand
    atoms are the alchemical ("removed", ss_alchemy = -2) species of the
    lambda windows; its bonded terms are those of polymer_in_water."""
    w = water_box(nwat=nwat, box=box, nfft=nfft, name="tmp")
    rng = np.random.default_rng(seed)
    lig = _grow_chain(nlig, rng)
    lig -= lig.mean(axis=0)
    wc = w.cartesian()
    keep = []
    for k in range(nwat):
        o = wc[:, 3 * k]
        d = lig - o
        d -= box * np.round(d / box)
        if (np.einsum("ij,ij->i", d, d) >= remove_within ** 2).all():
            keep.append(k)
    nw = len(keep)
    q = rng.normal(0.0, 0.35, nlig)
    lgroups = [(a, min(a + group_size - 1, nlig - 1)) for a in range(0, nlig, group_size)]
    for a, b in lgroups:
        q[a:b + 1] -= q[a:b + 1].mean()
    q -= q.mean()
    rl = np.random.default_rng(6)
    sig = rl.uniform(2.0, 3.8, NTYPE_CHAIN)
    eps = rl.uniform(0.02, 0.2, NTYPE_CHAIN)
    chain_types = [(s_ * 2.0 ** (1.0 / 6.0) / 2.0, e_) for s_, e_ in zip(sig, eps)]
    lt_lig = rng.integers(1, NTYPE_CHAIN + 1, nlig)
    n = nlig + 3 * nw
    pos = np.zeros((3, n))
    pos[:, :nlig] = lig.T
    for i, k in enumerate(keep):
        pos[:, nlig + 3 * i:nlig + 3 * i + 3] = wc[:, 3 * k:3 * k + 3]
    mass = np.concatenate([np.full(nlig, 12.011), np.tile([M_O, M_H, M_H], nw)])
    qa = np.concatenate([q, np.tile([Q_O, Q_H, Q_H], nw)])
    lt = np.concatenate([lt_lig, np.tile([NTYPE_CHAIN + 1, NTYPE_CHAIN + 2, NTYPE_CHAIN + 2], nw)]).astype(np.int32)
    groups = lgroups + [(nlig + 3 * i, nlig + 3 * i + 2) for i in range(nw)]
    molecules = [(0, nlig - 1)] + [(nlig + 3 * i, nlig + 3 * i + 2) for i in range(nw)]
    bonds = [(i, i + 1) for i in range(nlig - 1)]
    cons = []
    for i in range(nw):
        o = nlig + 3 * i
        for b in ((o, o + 1), (o, o + 2), (o + 1, o + 2)):
            bonds.append(b)
            cons.append(b)
    solute = np.zeros(n, dtype=bool)
    solute[:nlig] = True
    co = np.diag([box / 2.0] * 3)
    s = _assemble(name, co, pos, mass, qa, lt, chain_types + water_lj_types(), groups, molecules, bonds, solute,
                  constraints=cons, seed_v=4, alphal=0.35, order=4, nfft=tuple(nfft),
                  ncell=(max(3, int(box / 3.1)),) * 3, fudge=0.8333, lj_fudge=0.5)
    s.bond_k = np.full(len(s.bonds), 300.0 * 4184.0 / units.EFACT)
    s.bond_r0 = np.full(len(s.bonds), 1.53)
    s.bends = np.array([(i + 1, i + 2, i + 3) for i in range(nlig - 2)], dtype=np.int32)
    s.bend_k = np.full(len(s.bends), 60.0 * 4184.0 / units.EFACT)
    s.bend_t0 = np.full(len(s.bends), math.radians(112.0))
    s.tors = np.array([(i + 1, i + 2, i + 3, i + 4) for i in range(nlig - 3)], dtype=np.int32)
    s.tors_k = np.full(len(s.tors), 1.4 * 4184.0 / units.EFACT)
    s.tors_n = np.full(len(s.tors), -3.0)
    ss = np.ones(n, dtype=np.int32)
    ss[:nlig] = -2
    s.ss_alchemy = ss
    return s


def config3_window(k, nwin=64):
    """Lambda window k of the 64-window alchemical batch: the ligand system
    with lrm = lrmq = k / (nwin - 1) (soft core 0.5 0.5)."""
    s = ligand_in_water()
    s.name = f"ligand40_window{k}"
    return s, k / (nwin - 1)


def config2_polymer():
    return polymer_in_water()


# ------------------------------------------------- uneven solvated systems


def _smooth(n):
    for f in (2, 3, 5, 7):
        while n % f == 0:
            n //= f
    return n == 1


def pme_grid_for(box, spacing=1.0, lo=32, hi=96):
    """SPME grid points per axis for a cubic box: ceil(L / spacing) rounded up
    to the next size that factors into 2, 3, 5 and 7, clamped to [lo, hi]."""
    n = max(lo, int(math.ceil(box / spacing - 1e-9)))
    while not _smooth(n):
        n += 1
    return min(n, hi)


def linked_cells_for(box, shells, cell=3.1):
    """Cells per axis of a cubic box for the outer list radius (rcuth +
    rtolh + rneih): about `cell` A wide, and fine enough that the stencil
    reaches no cell twice (the check of src/lc_index.f:106-122: the widest
    offset floor(r / w) + 1 must stay below (n + 1) / 2)."""
    r = shells.rcuth + shells.rtolh + shells.rneih
    n0 = max(3, int(box / cell))
    for n in range(n0, 4 * n0 + 8):
        if int(r / (box / n)) + 1 < (n + 1) // 2:
            return n
    raise ValueError(f"box {box:.2f} A too small for linked cells at list radius {r:.2f} A")


def _rotations(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    a, b, c, d = q.T
    return np.stack([
        np.stack([a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)], axis=1),
        np.stack([2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)], axis=1),
        np.stack([2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d], axis=1),
    ], axis=1)


def _chain_lj_types():
    rl = np.random.default_rng(6)
    sig = rl.uniform(2.0, 3.8, NTYPE_CHAIN)
    eps = rl.uniform(0.02, 0.2, NTYPE_CHAIN)
    return [(s_ * 2.0 ** (1.0 / 6.0) / 2.0, e_) for s_, e_ in zip(sig, eps)]


def solvated_chains(natoms, seed, solute_frac=0.075, chain_len=100, density=0.100, group_size=3, name=None,
                    clash=2.2, remove_within=2.4, jitter=0.3, min_spacing=2.95):
    """A solute of bonded chains (built like the polymer: bond 1.53 A, angle
    112 deg, random torsions, charges N(0, 0.35) neutralised per group and
    per chain, LJ types of the polymer) in water, about `natoms` atoms in a
    cubic box sized for `density` atoms/A^3, SPME grid of about 1 A spacing
    (pme_grid_for).  The solute is round(solute_frac * natoms) atoms in
    chains of chain_len atoms (the last one takes the remainder), placed at
    random centres with no atom within `clash` A of an earlier chain; waters
    sit on a jittered cubic lattice, sites within `remove_within` A of a
    solute atom removed, the rest drawn at random.  Solute atoms are
    ss_index 1 (the rematom segment of the HREM replicas)."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    box = (natoms / density) ** (1.0 / 3.0)
    nsol = max(8, int(round(solute_frac * natoms)))
    lens = [chain_len] * (nsol // chain_len)
    rem = nsol - sum(lens)
    if rem >= 8 or not lens:
        lens.append(max(rem, 8))
    else:
        lens[-1] += rem
    nsol = sum(lens)
    nwat = (natoms - nsol) // 3
    # The water lattice is no denser than the liquid box's (spacing >=
    # min_spacing).  Where the volume the solute leaves cannot hold the
    # waters at that spacing, the box grows by 1% (density a little below
    # `density`) and the chains are placed again: a chain placed in a
    # smaller box can sit closer to another's periodic image in a larger one.
    while True:
        state = rng.bit_generator.state
        chains = []
        placed = np.zeros((0, 3))
        for n_c in lens:
            for _ in range(200):
                c = _grow_chain(n_c, rng, center=rng.uniform(-box / 2, box / 2, 3), clash=clash, box=box)
                if len(placed):
                    t = cKDTree(np.mod(placed + box / 2, box), boxsize=box)
                    if any(t.query_ball_point(np.mod(c + box / 2, box), clash, return_length=True)):
                        continue
                break
            else:
                raise RuntimeError("chain placement failed")
            chains.append(c)
            placed = np.concatenate([placed, c])
        tsol = cKDTree(np.mod(placed + box / 2, box), boxsize=box)
        nl = int(box / min_spacing)
        a = box / nl
        g = (np.stack(np.meshgrid(*(np.arange(nl),) * 3, indexing="ij"), -1).reshape(-1, 3) + 0.5) * a
        g = g + rng.uniform(-jitter, jitter, g.shape)
        free = tsol.query_ball_point(np.mod(g, box), remove_within, return_length=True) == 0
        if free.sum() >= nwat:
            break
        box *= 1.01
        rng.bit_generator.state = state
    sites = g[free]
    sites = sites[np.sort(rng.permutation(len(sites))[:nwat])] - box / 2
    R = _rotations(rng, nwat)
    tmpl = _water_template()
    wpos = sites[:, None, :] + np.einsum("wij,kj->wki", R, tmpl)  # [nwat, 3, 3]
    n = nsol + 3 * nwat
    pos = np.zeros((3, n))
    pos[:, :nsol] = np.concatenate(chains).T
    pos[:, nsol:] = wpos.reshape(-1, 3).T
    q = np.zeros(nsol)
    groups, molecules, bonds, bends, tors = [], [], [], [], []
    a0 = 0
    for n_c in lens:
        qc = rng.normal(0.0, 0.35, n_c)
        for a in range(0, n_c, group_size):
            b = min(a + group_size, n_c)
            qc[a:b] -= qc[a:b].mean()
            groups.append((a0 + a, a0 + b - 1))
        qc -= qc.mean()
        q[a0:a0 + n_c] = qc
        molecules.append((a0, a0 + n_c - 1))
        bonds += [(a0 + i, a0 + i + 1) for i in range(n_c - 1)]
        bends += [(a0 + i + 1, a0 + i + 2, a0 + i + 3) for i in range(n_c - 2)]
        tors += [(a0 + i + 1, a0 + i + 2, a0 + i + 3, a0 + i + 4) for i in range(n_c - 3)]
        a0 += n_c
    lt_sol = rng.integers(1, NTYPE_CHAIN + 1, nsol)
    mass = np.concatenate([np.full(nsol, 12.011), np.tile([M_O, M_H, M_H], nwat)])
    qa = np.concatenate([q, np.tile([Q_O, Q_H, Q_H], nwat)])
    lt = np.concatenate([lt_sol, np.tile([NTYPE_CHAIN + 1, NTYPE_CHAIN + 2, NTYPE_CHAIN + 2], nwat)]).astype(np.int32)
    wg = [(nsol + 3 * i, nsol + 3 * i + 2) for i in range(nwat)]
    groups += wg
    molecules += wg
    cons = []
    for i in range(nwat):
        o = nsol + 3 * i
        cons += [(o, o + 1), (o, o + 2), (o + 1, o + 2)]
    bonds += cons
    solute = np.zeros(n, dtype=bool)
    solute[:nsol] = True
    ng = pme_grid_for(box)
    nc = linked_cells_for(box, Shells())
    sysm = _assemble(name or f"chains{nsol}_water{nwat}", np.diag([box / 2.0] * 3), pos, mass, qa, lt,
                     _chain_lj_types() + water_lj_types(), groups, molecules, bonds, solute, constraints=cons,
                     seed_v=seed + 1, alphal=0.35, order=4, nfft=(ng, ng, ng), ncell=(nc, nc, nc),
                     fudge=0.8333, lj_fudge=0.5)
    sysm.bond_k = np.full(len(sysm.bonds), 300.0 * 4184.0 / units.EFACT)
    sysm.bond_r0 = np.full(len(sysm.bonds), 1.53)
    sysm.bends = np.array(bends, dtype=np.int32).reshape(-1, 3) + 0
    sysm.bend_k = np.full(len(sysm.bends), 60.0 * 4184.0 / units.EFACT)
    sysm.bend_t0 = np.full(len(sysm.bends), math.radians(112.0))
    sysm.tors = np.array(tors, dtype=np.int32).reshape(-1, 4) + 0
    sysm.tors_k = np.full(len(sysm.tors), 1.4 * 4184.0 / units.EFACT)
    sysm.tors_n = np.full(len(sysm.tors), -3.0)
    sysm.rematom = solute.astype(np.uint8)
    return sysm


def uneven_specs(n=128, seed=9, lo=3000, hi=60000, seed_scale=10):
    """The uneven HREM batch: n systems with atom counts log-uniform in
    [lo, hi] and solute fractions U[0.05, 0.10] (seed), each with a solute
    scaling factor U[0.3, 1.0] (seed_scale) applied as rem_factor to the
    pairs touching the solute (seg_select kind 0)."""
    r = np.random.default_rng(seed)
    nat = np.exp(r.uniform(math.log(lo), math.log(hi), n)).round().astype(int)
    frac = r.uniform(0.05, 0.10, n)
    scale = np.random.default_rng(seed_scale).uniform(0.3, 1.0, n)
    return [dict(natoms=int(nat[k]), solute_frac=float(frac[k]), rem_factor=float(scale[k]), seed=1000 + k,
                 name=f"uneven{k}") for k in range(n)]


def build_spec(spec):
    """System of one uneven_specs entry (module-level so a process pool can
    map it)."""
    return solvated_chains(spec["natoms"], spec["seed"], spec["solute_frac"], name=spec["name"])


# -------------------------------------------------------------- small cases


def two_waters(sep=(3.0, 0.0, 0.0), box=20.0, across_face=False, seed=11):
    """Two waters (two groups) at a chosen COM separation; with across_face
    the pair straddles the periodic boundary along x."""
    rng = np.random.default_rng(seed)
    tmpl = _water_template()
    c0 = np.array([box / 2 - 0.5 * sep[0], 0.0, 0.0]) if across_face else np.zeros(3)
    c1 = c0 + np.array(sep)
    pos = np.zeros((3, 6))
    for w, c in enumerate((c0, c1)):
        R = _random_rotation(rng)
        for k in range(3):
            pos[:, 3 * w + k] = c + R @ tmpl[k]
    if across_face:
        # wrap the second molecule as a whole into the box
        shift = box * np.round(pos[:, 3:6].mean(axis=1) / box)
        pos[:, 3:6] -= shift[:, None]
    mass = np.tile([M_O, M_H, M_H], 2)
    q = np.tile([Q_O, Q_H, Q_H], 2)
    lt = np.tile([1, 2, 2], 2)
    groups = [(0, 2), (3, 5)]
    bonds = [(0, 1), (0, 2), (1, 2), (3, 4), (3, 5), (4, 5)]
    co = np.diag([box / 2.0] * 3)
    return _assemble("two_waters", co, pos, mass, q, lt, water_lj_types(), groups, groups, bonds,
                     np.zeros(6, dtype=bool), constraints=bonds, nfft=(16, 16, 16), ncell=(4, 4, 4))


def ion_pair_box(charges=(1.0, -1.0), pos=((0, 0, 0), (2.5, 0, 0)), box=16.0, nfft=(16, 16, 16)):
    """Single-atom groups (ions); no exclusions, LJ on both."""
    p = np.array(pos, dtype=float).T
    n = p.shape[1]
    mass = np.full(n, 22.99)
    lt = np.ones(n, dtype=np.int32)
    groups = [(i, i) for i in range(n)]
    co = np.diag([box / 2.0] * 3)
    return _assemble("ions", co, p, mass, list(charges), lt, [(1.5, 0.1)], groups, groups, [],
                     np.zeros(n, dtype=bool), nfft=tuple(nfft), ncell=(4, 4, 4))


def nacl_crystal(ncell=2, a=5.64, nfft=(32, 32, 32), alphal=None):
    """Rock-salt lattice of unit charges: the Ewald known answer (Madelung
    constant 1.747565 for the nearest-neighbour distance a/2)."""
    pts = []
    qs = []
    for i in range(2 * ncell):
        for j in range(2 * ncell):
            for k in range(2 * ncell):
                pts.append(((i + 0.25) * a / 2, (j + 0.25) * a / 2, (k + 0.25) * a / 2))
                qs.append(1.0 if (i + j + k) % 2 == 0 else -1.0)
    box = ncell * a
    p = np.array(pts).T - box / 2
    n = p.shape[1]
    mass = np.full(n, 22.99)
    lt = np.ones(n, dtype=np.int32)
    groups = [(i, i) for i in range(n)]
    co = np.diag([box / 2.0] * 3)
    s = _assemble("nacl", co, p, mass, qs, lt, [(0.0, 0.0)], groups, groups, [], np.zeros(n, dtype=bool),
                  nfft=tuple(nfft), ncell=(3, 3, 3))
    if alphal is not None:
        s.alphal = alphal
    return s
