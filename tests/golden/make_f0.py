"""Builds tests/golden/f0_fkbp12.npz, the real-system fixture "F0": the
solvated FKBP12-ligand system of the reference's test1/test2 (14,900 atoms,
5,082 groups, 90 LJ types) as ORAC assembled it (test1/1j4i.tpgprm, the
topology-parameter file ORAC wrote) at the state of a restart file ORAC
wrote (test2/b-RSTRT/ij4i0000.rst, step 30).  Only the arrays the force
path needs are kept, in the files' own units and 1-based indices;
orac_b200.oracio.system_from_orac turns them into a System.

Run from the repository root where the reference checkout is present:
    python tests/golden/make_f0.py [reference root]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "orac-porting_b200"))
from orac_b200 import oracio  # noqa: E402

KEYS_INT = ("ss_index", "nbtype", "grppt", "lbnd", "lbndg", "ltor", "litr", "int14", "type14", "int13", "mapnl")
KEYS_F = ("chrge", "mass", "potbo", "potbe", "potto", "potit", "pnbd")
DEFAULT_ROOT = "/root/reference"
SCALARS = ("ntap", "ngrp", "lbond", "lbend", "ltors", "litor", "lpnbd", "int14p", "int13p", "nmapnl", "iz")


def build_arrays(root):
    tp = oracio.read_tpgprm(os.path.join(root, "test1", "1j4i.tpgprm"))
    rs = oracio.read_rst(os.path.join(root, "test2", "b-RSTRT", "ij4i0000.rst"), tp["ntap"])
    out = {k: np.asarray(tp[k], dtype=np.int32) for k in KEYS_INT}
    out.update({k: np.asarray(tp[k], dtype=np.float64) for k in KEYS_F})
    out.update({k: np.array(tp[k]) for k in SCALARS})
    out.update(co=rs["co"], xyz=rs["xyz"], v=rs["v"], nstep=np.array(rs["nstep"]))
    return out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_ROOT
    arrs = build_arrays(root)
    path = os.path.join(HERE, "f0_fkbp12.npz")
    np.savez_compressed(path, **arrs)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
