"""Builds tests/golden/ne_test4.npz: the non-equilibrium alchemy run of the
reference's test4 (the FKBP12 ligand, atoms 1-52, switched off along the
schedule test4/15.off with the shifted potential, four walkers started
from test2's restart files): the schedule (times in ps, ladded laddedq
lremoved lremovedq, the file's columns) and, per walker, the work file ORAC
wrote (PAR000k/1.5.wrk: time in ps, lambda-added LJ and QQ, lambda-removed
LJ and QQ, work in kJ/mol).

Run from the repository root with the path of a reference checkout:
    python tests/golden/make_ne_test4.py <reference root>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_table(path):
    rows = []
    for line in open(path):
        t = line.split()
        if not t or t[0].startswith("#"):
            continue
        rows.append([float(x) for x in t])
    return np.array(rows)


def main(root):
    t4 = os.path.join(root, "test4")
    sched = read_table(os.path.join(t4, "15.off"))
    out = {"schedule": sched}
    for k in range(1, 5):
        out[f"wrk{k}"] = read_table(os.path.join(t4, f"PAR000{k}", "1.5.wrk"))
    np.savez(os.path.join(HERE, "ne_test4.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
