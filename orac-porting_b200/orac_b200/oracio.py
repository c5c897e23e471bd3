"""ORAC's topology-parameter and restart files.

ORAC writes its assembled system (`WRITE_TPGPRM`, src/dumptp.f) and its MD
state (`RESTART write`, src/dumprs.f) as Fortran list-directed ASCII; it
reads them back with src/readtp.f and src/readrs.f.  This module reads
both, converts the topology to ORAC's program units the way ORAC does
after reading (src/covchg.f, src/covbd.f, src/covnb.f, src/setup_box.f
:412-434), builds a `systems.System` from them, and writes restart files in
the layout ORAC reads, so a real ORAC system can be run here and its state
handed back.

List-directed records: each Fortran READ statement starts at a new record
(line), takes as many values as its list needs across lines, and skips the
rest of its last line; a READ with an empty list still consumes one line.
`_Records` follows these rules.
"""
from __future__ import annotations

import math

import numpy as np

from . import units


class _Records:
    def __init__(self, path):
        with open(path) as f:
            self.lines = f.read().split("\n")
        self.pos = 0

    def read(self, n):
        """The next n values of one READ statement (strings)."""
        out = []
        if n == 0:
            self.pos += 1
            return out
        while len(out) < n:
            if self.pos >= len(self.lines):
                raise EOFError("end of file inside a record")
            for tok in self.lines[self.pos].replace(",", " ").split():
                if "*" in tok:  # r*c repeat count
                    r, c = tok.split("*", 1)
                    out.extend([c] * int(r))
                else:
                    out.append(tok)
            self.pos += 1
        return out[:n]  # the rest of the last record is skipped

    def ints(self, n):
        return np.array([int(t) for t in self.read(n)], dtype=np.int64)

    def floats(self, n):
        return np.array([float(t.replace("D", "E").replace("d", "e")) for t in self.read(n)], dtype=np.float64)


def _logical(t):
    return t.strip().upper().lstrip(".").startswith("T")


def read_tpgprm(path, amphi=False):
    """The topology-parameter file in src/readtp.f's order.  Arrays keep
    ORAC's 1-based indices and the file's units (charges in e, energies in
    kcal/mol, angles in degrees)."""
    r = _Records(path)
    h = r.read(23)
    names = ("llacc", "lldon", "nbone", "ntap", "lbond", "lbend", "ltors", "litor", "lpnbd", "int14p", "int13p",
             "nspw", "nunit", "lphyd", "ngrp", "nrigg", "nrigat", "nmapnl", "nmol", "nato_slv")
    d = {k: int(v) for k, v in zip(names, h[:20])}
    d["adihed"], d["slv_exist"], d["slt_exist"] = (_logical(t) for t in h[20:23])
    N, G, nb, na, nt, ni, npot = d["ntap"], d["ngrp"], d["lbond"], d["lbend"], d["ltors"], d["litor"], d["lpnbd"]
    sp = r.ints(2)
    d["ss_point"] = r.ints(int(sp[0]) + int(sp[1]))
    d["ss_index"] = r.ints(N)
    r.ints(2 * d["llacc"] + 2 * d["lldon"])  # H-bond acceptors and donors
    d["nbtype"] = r.ints(N)
    d["nres1"] = r.ints(N)
    d["nres2"] = r.ints(N)
    d["mback"] = r.ints(N)
    g = r.ints(2 * G)
    d["grppt"] = np.stack([g[:G], g[G:]], axis=1)
    b = r.ints(2 * nb)
    d["lbnd"] = np.stack([b[:nb], b[nb:]], axis=1)
    # connection table: per atom a count and that many neighbours, one READ
    conn, buf = [], []
    while len(conn) < N:
        while not buf:
            buf = r.lines[r.pos].split()
            r.pos += 1
        k = int(buf.pop(0))
        while len(buf) < k:
            buf += r.lines[r.pos].split()
            r.pos += 1
        conn.append([int(x) for x in buf[:k]])
        buf = buf[k:]
    if buf:
        raise ValueError("connection table record longer than its counts")
    d["concta"] = conn
    d["lbndg"] = r.ints(3 * na).reshape(3, na).T
    d["ltor"] = r.ints(4 * nt).reshape(4, nt).T
    d["litr"] = r.ints(4 * ni).reshape(4, ni).T
    n14, n13 = d["int14p"], d["int13p"]
    v = r.read(2 * n14 + n14 + 2 * n13 + npot * npot)
    o = 0
    d["int14"] = np.array(v[o:o + 2 * n14], dtype=np.int64).reshape(n14, 2)
    o += 2 * n14
    d["type14"] = np.array(v[o:o + n14], dtype=np.int64)
    o += n14
    d["int13"] = np.array(v[o:o + 2 * n13], dtype=np.int64).reshape(n13, 2)
    o += 2 * n13
    d["nhtype"] = np.array(v[o:], dtype=np.int64).reshape(npot, npot)
    v = r.floats(1 + 2 * N)
    d["wmtp"], d["chrge"], d["mass"] = v[0], v[1:1 + N], v[1 + N:]
    d["mapnl"] = r.ints(d["nmapnl"])
    nbun, iz = r.ints(2)
    d["nbun"], d["iz"] = int(nbun), int(iz)
    ntc = 4 if amphi else 2
    lp = d["lphyd"]
    cnt = 2 * nb + 7 * na + ntc * nt + 3 * ni + 4 * npot + (2 * npot if amphi else 0) + 2 * lp
    v = r.floats(cnt)
    o = 0

    def take(n, w):
        nonlocal o
        a = v[o:o + n * w].reshape(w, n).T.copy()  # ((p(i,j),i=1,n),j=1,w)
        o += n * w
        return a

    d["potbo"] = take(nb, 2)
    d["potbe"] = take(na, 7)
    d["potto"] = take(nt, ntc)
    d["potit"] = take(ni, 3)
    d["pnbd"] = take(npot, 4)  # pnbd1..pnbd4 as columns
    if amphi:
        d["sjorg"], d["ejorg"] = take(npot, 1)[:, 0], take(npot, 1)[:, 0]
    if iz == 1:
        m = npot * (npot + 1) // 2
        e = r.floats(2 * m)
        d["ecc6_file"], d["ecc12_file"] = e[:m], e[m:]
    return d


def read_rst(path, ntap=None):
    """An ORAC restart file (src/readrs.f:216-236): box co and oc, step and
    temperature, sizes, Cartesian positions and velocities."""
    r = _Records(path)
    v = r.floats(18)
    co = v[:9].reshape(3, 3)  # ((co(i,j),j=1,3),i=1,3): row by row
    oc = v[9:].reshape(3, 3)
    t = r.read(2)
    nstep, temp = int(t[0]), float(t[1].replace("D", "E"))
    n, ngrp, nprot = (int(x) for x in r.read(3))
    if ntap is not None and n != ntap:
        raise ValueError(f"restart holds {n} atoms, the topology {ntap}")
    big = r.floats(6 * n + 3 * ngrp + 6 * nprot)
    x = big[:3 * n].reshape(3, n)
    vel = big[3 * n:6 * n].reshape(3, n)
    out = dict(co=co, oc=oc, nstep=nstep, temp=temp, ntap=n, ngrp=ngrp, nprot=nprot, xyz=x, v=vel)
    # the thermostats' state when the run had them (src/readrs.f:240-251:
    # vpx1, the averages, then hoover and cpress, and with hoover nh, gh =
    # eta, vh = etap, vh1); older or shorter files end before it
    try:
        r.floats(3 * n)
        n1, n2 = (int(v) for v in r.read(2))
        r.floats(n1 + n2)
        hoover = r.read(2)[0].upper().startswith(("T", ".T"))
        if hoover:
            nh = int(r.read(1)[0])
            g = r.floats(3 * nh)
            out["eta"], out["etap"] = g[:nh].copy(), g[nh:2 * nh].copy()
    except (EOFError, ValueError, IndexError):
        pass
    return out


def write_rst(path, co, xyz, v, nstep=0, temp=0.0, grp=None, ngrp=0, mol=None, nprot=0, thermostat=None):
    """A restart file with the records ORAC reads (src/readrs.f:216-251):
    box, step and temperature, sizes, positions, velocities (twice, as
    src/dumprs.f writes vpx and vpx1), group and molecule centres (zero when
    not given), no running averages, no barostat state; thermostat = (eta,
    etap) of the three Nose-Hoover thermostats writes hoover and ORAC's gh,
    vh and vh1 records (vh1 as etap)."""
    co = np.asarray(co, dtype=np.float64)
    oc = np.linalg.inv(co)
    n = xyz.shape[1]
    grp = np.zeros((3, ngrp)) if grp is None else np.asarray(grp)
    mol = np.zeros((3, nprot)) if mol is None else np.asarray(mol)

    def rec(vals):
        return " ".join(repr(float(x)) if not isinstance(x, (int, np.integer)) else str(int(x)) for x in vals) + "\n"

    with open(path, "w") as f:
        f.write(rec(list(co.ravel()) + list(oc.ravel())))
        f.write(f"{int(nstep)} {float(temp)!r}\n")
        f.write(f"{n} {ngrp} {nprot}\n")
        f.write(rec(np.concatenate([xyz.ravel(), v.ravel(), grp.ravel(), mol.ravel(), np.zeros(3 * nprot)])))
        f.write(rec(v.ravel()))
        f.write("0 0\n\n")
        if thermostat is None:
            f.write("F F\n")
        else:
            eta, etap = (np.asarray(t, dtype=np.float64).ravel() for t in thermostat)
            f.write("T F\n")
            f.write(f"{len(eta)}\n")
            f.write(rec(np.concatenate([eta, etap, etap])))
        f.write("F\n")


def _components(n, pairs):
    """Connected components of the bond graph (0-based labels by first atom)."""
    parent = np.arange(n)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for a, b in pairs:
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    roots = np.array([find(a) for a in range(n)])
    _, lab = np.unique(roots, return_inverse=True)
    return lab


def system_from_orac(tp, rst, alphal, nfft, order, shells, ncell, fudge=0.83333, lj_fudge=0.5, name="orac",
                     rigid_hydrogen=False, move_fast_torsions=True):
    """A System from read_tpgprm / read_rst output with ORAC's conversions:
    charges to program units (src/covchg.f), bonded parameters (src/covbd.f:
    force constants from kcal/mol, angles of bends and harmonic impropers to
    radians), LJ tables by the amber mixing rule from the per-type
    parameters (src/covnb.f, iz = 0) with the 1-4 tables from their own
    parameters or, where those vanish, lj_fudge times the regular ones.
    Molecules are the connected components of the bond list.  Constraints
    are an MD-input choice, not part of the file: every bond is flexible,
    or with rigid_hydrogen every bond to a hydrogen (mass below 1.5 amu) is
    a constraint at its force-field length (ORAC's `STRETCHING HEAVY` with
    the bond lengths adjusted to the force field) and leaves the bond
    list.  With move_fast_torsions (ORAC's default) the fast proper
    torsions become cosine impropers as ORAC's MD driver makes them
    (fast_torsions)."""
    from . import systems

    N, G = tp["ntap"], tp["ngrp"]
    if tp["iz"] != 0:
        raise NotImplementedError("topology without mixing rules (iz = 1)")
    kconv = 4184.0 / units.EFACT
    co = np.asarray(rst["co"], dtype=np.float64)
    xyz = np.asarray(rst["xyz"], dtype=np.float64)
    scaled = np.linalg.inv(co) @ xyz
    grppt = tp["grppt"].astype(np.int32)
    atomg = np.zeros(N, dtype=np.int32)
    for g, (a, b) in enumerate(grppt):
        atomg[a - 1:b] = g + 1
    mol = _components(N, [(a - 1, b - 1) for a, b in tp["lbnd"]])
    atomp = (mol + 1).astype(np.int32)
    mass = tp["mass"].astype(np.float64)
    gm = np.bincount(atomg - 1, weights=mass)
    pmass = mass / gm[atomg - 1]
    npot = tp["lpnbd"]
    pn = tp["pnbd"]
    fact = 1.0 / (2.0 ** (1.0 / 6.0))
    e12 = np.zeros(npot * (npot + 1) // 2)
    e6 = np.zeros_like(e12)
    e1412 = np.zeros_like(e12)
    e146 = np.zeros_like(e12)
    tt = np.zeros((npot, npot), dtype=np.int32)
    for i in range(npot):
        for j in range(i, npot):
            ij = (j + 1) * j // 2 + i  # 0-based of ORAC's j*(j-1)/2 + i
            tt[i, j] = tt[j, i] = ij + 1
            qe = math.sqrt(abs(pn[i, 1] * pn[j, 1])) * 4.0 * kconv
            s6 = ((pn[i, 0] + pn[j, 0]) * fact) ** 6
            e6[ij], e12[ij] = qe * s6, qe * s6 * s6
            q4 = math.sqrt(abs(pn[i, 3] * pn[j, 3])) * 4.0 * kconv
            s46 = ((pn[i, 2] + pn[j, 2]) * fact) ** 6
            e146[ij], e1412[ij] = q4 * s46, q4 * s46 * s46
            if abs(e1412[ij]) < 1e-12:
                e146[ij], e1412[ij] = e6[ij] * lj_fudge, e12[ij] * lj_fudge
    # non-excluded pairs inside a group (fnbgrp's list, built by ORAC at set-up)
    mapnl = tp["mapnl"].astype(np.int32)
    excl = [set() for _ in range(N)]
    p = 0
    for a in range(N):
        k = int(mapnl[p])
        excl[a].update(int(x) - 1 for x in mapnl[p + 1:p + 1 + k])
        p += k + 1
    ingrp = [(i + 1, j + 1) for a, b in grppt for i in range(a - 1, b) for j in range(i + 1, b) if j not in excl[i]]
    lb = tp["lbnd"]
    flex = np.ones(len(lb), dtype=bool)
    if rigid_hydrogen:
        flex = ~((mass[lb[:, 0] - 1] < 1.5) | (mass[lb[:, 1] - 1] < 1.5))
    be = tp["potbe"].copy()
    it = tp["potit"].copy()
    sysm = systems.System(
        name=name, ntap=N, ngrp=G, nprot=int(atomp.max()), co=co,
        xp0=scaled[0].copy(), yp0=scaled[1].copy(), zp0=scaled[2].copy(), mass=mass,
        charge=np.array([units.charge_internal(q) for q in tp["chrge"]]), nbtype=tp["nbtype"].astype(np.int32),
        ntype=npot, type_table=tt, ecc12=e12, ecc6=e6, grppt=grppt, atomg=atomg, atomp=atomp,
        ss_index=tp["ss_index"].astype(np.int32), pmass=pmass, mapnl=mapnl,
        int14=tp["int14"].astype(np.int32).reshape(-1, 2), type14=tp["type14"].astype(np.int32),
        ecc1412=e1412, ecc146=e146, ingrp=np.array(ingrp, dtype=np.int32).reshape(-1, 2),
        bonds=tp["lbnd"][flex].astype(np.int32), bend13=tp["int13"].astype(np.int32).reshape(-1, 2),
        constraints=tp["lbnd"][~flex].astype(np.int32), cdist=tp["potbo"][~flex, 1].copy(),
        vx=rst["v"][0].copy(), vy=rst["v"][1].copy(), vz=rst["v"][2].copy(),
        alphal=alphal, order=order, nfft=tuple(nfft), shells=shells, fudge=fudge, lj_fudge=lj_fudge,
        ncell=tuple(ncell), lj_params=pn[:, :2].copy(),
    )
    # src/covbd.f: energies from kcal/mol, angles from degrees
    sysm.bond_k = tp["potbo"][flex, 0] * kconv
    sysm.bond_r0 = tp["potbo"][flex, 1].copy()
    sysm.bends = tp["lbndg"].astype(np.int32)
    sysm.bend_t0 = np.radians(be[:, 1])
    sysm.bend_k = be[:, 0] * kconv
    sysm.bend_ub_r0 = be[:, 3].copy()
    sysm.bend_ub_k = be[:, 2] * kconv
    ltor, litr, to = tp["ltor"], tp["litr"], tp["potto"]
    fast = fast_torsions(ltor, to, mass) if move_fast_torsions else np.zeros(len(ltor), dtype=bool)
    sysm.tors = ltor[~fast].astype(np.int32)
    sysm.tors_k = to[~fast, 0] * kconv
    sysm.tors_n = to[~fast, 1].copy()
    # moved torsions follow the file's impropers as cosine impropers (c = -1)
    sysm.itors = np.concatenate([litr, ltor[fast]]).astype(np.int32)
    sysm.itors_b = np.concatenate([it[:, 0], to[fast, 0]]) * kconv
    sysm.itors_a = np.concatenate([np.where(it[:, 2] > 0.0, np.radians(it[:, 1]), it[:, 1]), to[fast, 1]])
    sysm.itors_c = np.concatenate([it[:, 2], np.full(int(fast.sum()), -1.0)])
    return sysm


def fast_torsions(ltor, potto, mass):
    """ORAC's run-time move of "fast" proper torsions into the improper
    list (src/mtsmd.f:990-1030, on unless the integrator input says
    `no_adjust_itors`): a torsion whose uncoupled frequency
    sqrt(tfactor k / mu) n / (2 pi c) exceeds 300 cm^-1 is evaluated by
    fitors as a cosine improper (potc = -1) at the fastest intramolecular
    level instead of by fptors.  k is the barrier in kcal/mol, n the signed
    multiplicity (a negative n never moves), mu = (m1 + m4) sin^2(60 deg)
    with m = 1 for an end atom whose type name starts with "h" and 12
    otherwise; the file carries masses, not type names, and here a
    hydrogen is an atom below 1.5 amu.  The literals keep ORAC's
    precisions (0.001 and 3.14 are single-precision constants in the
    Fortran).  Returns a mask over the torsions."""
    tfactor = 4.0 * 4.184e3 * 1.0e20 / float(np.float32(0.001))
    m1 = np.where(mass[ltor[:, 0] - 1] < 1.5, 1.0, 12.0)
    m4 = np.where(mass[ltor[:, 3] - 1] < 1.5, 1.0, 12.0)
    xmu = (m1 + m4) * math.sin(3.14 / 3.0) ** 2
    naux = np.rint(potto[:, 1])
    freq = np.sqrt(tfactor * np.abs(potto[:, 0]) / xmu) * naux / (3.0e10 * 2 * float(np.float32(3.14)))
    return freq > 300.0


def split_arrays(arrs):
    """(topology, restart) dicts for system_from_orac from one mapping of
    arrays holding read_tpgprm's and read_rst's fields (a saved fixture)."""
    tp = {k: (int(arrs[k]) if np.ndim(arrs[k]) == 0 else np.asarray(arrs[k])) for k in arrs
          if k not in ("co", "xyz", "v", "nstep")}
    rst = dict(co=np.asarray(arrs["co"]), xyz=np.asarray(arrs["xyz"]), v=np.asarray(arrs["v"]),
               nstep=int(arrs["nstep"]))
    return tp, rst


def load(tpgprm_path, rst_path, **kw):
    """A System from ORAC's own files: a topology-parameter file (as ORAC's
    WRITE_TPGPRM writes it) and a restart file, with the run parameters of
    system_from_orac as keywords (alphal, nfft, order, shells, ncell, ...)."""
    tp = read_tpgprm(tpgprm_path)
    return system_from_orac(tp, read_rst(rst_path, tp["ntap"]), **kw)


def write_system_rst(path, s, x, v, nstep=0):
    """An ORAC restart file of System `s` at Cartesian positions x and
    velocities v (3, N): the box, the step count, the kinetic temperature
    (3N minus the constraints minus the three of the centre of mass), and
    the group and molecule centres of mass that ORAC's restart carries."""
    x = np.asarray(x, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    mass = np.asarray(s.mass, dtype=np.float64)
    ekin = 0.5 * float((mass * (v * v).sum(0)).sum())
    ndf = 3 * s.ntap - len(np.asarray(s.constraints).reshape(-1, 2)) - 3
    temp = units.kinetic_temperature(ekin, ndf) if ndf > 0 else 0.0
    g = np.asarray(s.atomg) - 1
    grp = np.zeros((3, s.ngrp))
    for d in range(3):
        grp[d] = np.bincount(g, weights=np.asarray(s.pmass) * x[d], minlength=s.ngrp)
    p = np.asarray(s.atomp) - 1
    mt = np.bincount(p, weights=mass, minlength=s.nprot)
    mol = np.stack([np.bincount(p, weights=mass * x[d], minlength=s.nprot) / mt for d in range(3)])
    write_rst(path, s.co, x, v, nstep=nstep, temp=temp, grp=grp, ngrp=s.ngrp, mol=mol, nprot=s.nprot)
