"""Builds tests/golden/f0_fkbp12.npz, the real-system fixture "F0": the
solvated FKBP12-ligand system of the reference's test1/test2 (14,900 atoms,
5,082 groups, 90 LJ types) as ORAC assembled it (test1/1j4i.tpgprm, the
topology-parameter file ORAC wrote) at the state of a restart file ORAC
wrote (test2/b-RSTRT/ij4i0000.rst, step 30).  Only the arrays the force
path needs are kept, in the files' own units and 1-based indices;
orac_b200.oracio.system_from_orac turns them into a System.

Also builds tests/golden/f0_orac_records.npz: the positions, velocities and
boxes of test2's other two replica-1 restart files (ij4i0001.rst,
ij4i0003.rst) and, for all three states, the Nose-Hoover thermostats'
state the restart carries and the energy record ORAC printed at the step it
wrote the restart (test2/PAR0001/out0001, matched by box edge and
temperature).

Run from the repository root with the path of a reference checkout:
    python tests/golden/make_f0.py <reference root>
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "orac-porting_b200"))
from orac_b200 import oracio  # noqa: E402

KEYS_INT = ("ss_index", "nbtype", "grppt", "lbnd", "lbndg", "ltor", "litr", "int14", "type14", "int13", "mapnl")
KEYS_F = ("chrge", "mass", "potbo", "potbe", "potto", "potit", "pnbd")
SCALARS = ("ntap", "ngrp", "lbond", "lbend", "ltors", "litor", "lpnbd", "int14p", "int13p", "nmapnl", "iz")


def build_arrays(root):
    tp = oracio.read_tpgprm(os.path.join(root, "test1", "1j4i.tpgprm"))
    rs = oracio.read_rst(os.path.join(root, "test2", "b-RSTRT", "ij4i0000.rst"), tp["ntap"])
    out = {k: np.asarray(tp[k], dtype=np.int32) for k in KEYS_INT}
    out.update({k: np.asarray(tp[k], dtype=np.float64) for k in KEYS_F})
    out.update({k: np.array(tp[k]) for k in SCALARS})
    out.update(co=rs["co"], xyz=rs["xyz"], v=rs["v"], nstep=np.array(rs["nstep"]))
    return out


# columns of ORAC's energy record (src/prtacc.f, format 12002) kept for the
# states of the restart files, in kJ/mol (TotTemp in K)
RECORD_KEYS = ("SlvNonbd", "SlvCoul", "SltCoul", "SltL-J", "SltBond", "SltStr", "SltBen", "SltItor", "SltPtor",
               "S-SPot", "S-SCoul", "TotTemp")
RESTARTS = ("ij4i0000.rst", "ij4i0001.rst", "ij4i0003.rst")


def parse_records(path):
    """Every energy record of an ORAC output: (box edge from the XYZ line
    that follows it, {column: value}, line number)."""
    lines = open(path).read().splitlines()
    out, cur = [], None
    for k, line in enumerate(lines):
        if "Tstep    =" in line:
            cur = ({}, k + 1)
        if cur is not None:
            for key, val in re.findall(r"(\S+)\s*=\s*(-?[\d.]+)", line):
                cur[0].setdefault(key, float(val))
            if line.startswith(" XYZ"):
                out.append((float(line.split()[1]), cur[0], cur[1]))
                cur = None
    return out


def build_records(root, ntap):
    """The replica-1 states that test2 saved as restart files with the
    energy record ORAC printed for the same step (matched by box edge and
    temperature): positions, velocities and box of each, and the record's
    columns."""
    recs = parse_records(os.path.join(root, "test2", "PAR0001", "out0001"))
    out = {"keys": np.array(RECORD_KEYS), "restarts": np.array(RESTARTS)}
    vals, where = [], []
    for k, name in enumerate(RESTARTS):
        rs = oracio.read_rst(os.path.join(root, "test2", "b-RSTRT", name), ntap)
        edge = 2.0 * rs["co"][0, 0]
        hit = [(d, ln) for e, d, ln in recs if abs(e - edge) < 6e-5 and abs(d["TotTemp"] - rs["temp"]) < 6e-3]
        if len(hit) != 1:
            raise RuntimeError(f"{name}: {len(hit)} matching records")
        d, ln = hit[0]
        vals.append([d[c] for c in RECORD_KEYS])
        where.append(ln)
        if k > 0:  # the first state is f0_fkbp12.npz's own
            out[f"co{k}"] = rs["co"]
            out[f"xyz{k}"] = rs["xyz"]
            out[f"v{k}"] = rs["v"]
        # the three Nose-Hoover thermostats' coordinates and velocities the
        # restart carries (src/readrs.f:247-251: gh, vh)
        out[f"eta{k}"] = rs["eta"]
        out[f"etap{k}"] = rs["etap"]
    out["printed"] = np.array(vals)
    out["out0001_line"] = np.array(where)
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_f0.py <reference root>")
    root = sys.argv[1]
    arrs = build_arrays(root)
    path = os.path.join(HERE, "f0_fkbp12.npz")
    np.savez_compressed(path, **arrs)
    print(path, os.path.getsize(path), "bytes")
    recs = build_records(root, int(arrs["ntap"]))
    path = os.path.join(HERE, "f0_orac_records.npz")
    np.savez_compressed(path, **recs)
    print(path, os.path.getsize(path), "bytes", "records at out0001 lines", list(recs["out0001_line"]))


if __name__ == "__main__":
    main()
