"""The oracle's restatement of ORAC's intra-alchemical corrections:
fnb14_alchemy (src/fnb14_alchemy.f:225-341) and ferrf_alchemy_add over
listqq (src/ferrf_alchemy_add.f, src/initialize_lambda.f:62-139).

- listqq holds every pair of alchemical atoms that is no bond, constraint,
  1-3 or 1-4 pair, with facQ 1 for one species and 0 across species;
- forces are minus the gradient of the energies (central differences);
- what the corrections are for: a removed ligand's own Coulomb stays at
  full strength whatever lambda.  For a listqq pair the direct lattice's
  Q Q erfc/r, the scaled reciprocal sum's (1-l)^2 Q Q erf/r and
  ferrf_alchemy_add add up to Q Q / r; for a 1-4 pair fnb14_alchemy's terms,
  the reciprocal (1-l)^2 Q Q erf/r and ferrf's -(1-f)(1-l)^2 Q Q erf/r add
  up to f Q Q / r.
"""
import numpy as np
import pytest

import oracle
from orac_b200 import systems


def ligand():
    return systems.ligand_in_water()


def test_listqq_is_the_alchemical_pairs_beyond_1_4():
    s = ligand()
    o = oracle.Oracle(s.copy())
    lst = o.alch_listqq(s.ss_alchemy)
    al = np.where(np.abs(s.ss_alchemy) == 2)[0] + 1
    excl = set()
    for a in (s.bonds, s.constraints, s.bend13, s.int14):
        for i, j in np.asarray(a).reshape(-1, 2):
            excl.add((min(i, j), max(i, j)))
    want = {(min(i, j), max(i, j)) for k, i in enumerate(al) for j in al[k + 1:]} - excl
    got = {(min(i, j), max(i, j)) for i, j, _ in lst}
    assert got == want and len(got) == len(lst)
    assert np.all(lst[:, 2] == 1)  # one species (all removed)


def _energy(o, s, lam, which):
    lq = o.alch_lambdas(s.ss_alchemy, 0.0, lam)
    if which == "add":
        return o.ferrf_alchemy_add(o.alch_listqq(s.ss_alchemy), lq)
    return o.fnb14_alchemy(lq, lq)


@pytest.mark.parametrize("which", ["add", "14"])
def test_forces_are_minus_the_gradient(which):
    s = ligand()
    o = oracle.Oracle(s.copy())
    F, e, _ = _energy(o, s, 0.35, which)
    al = np.where(np.abs(s.ss_alchemy) == 2)[0][:6]
    h = 1e-6
    for a in al:
        for d in range(3):
            us = []
            for sg in (1, -1):
                t = s.copy()
                x = t.cartesian()
                x[d, a] += sg * h
                sc = np.linalg.inv(t.co) @ x
                t.xp0, t.yp0, t.zp0 = sc[0], sc[1], sc[2]
                us.append(_energy(oracle.Oracle(t), t, 0.35, which)[1].sum())
            fd = -(us[0] - us[1]) / (2 * h)
            assert abs(F[d, a] - fd) <= 1e-6 * max(1.0, abs(fd)), (a, d, F[d, a], fd)


def test_ligand_coulomb_stays_whole():
    """Per pair, at lambda 0.6: direct + scaled reciprocal + corrections =
    the full Coulomb of the pair (fudged for 1-4 pairs)."""
    s = ligand()
    o = oracle.Oracle(s.copy())
    lam = 0.6
    lq = o.alch_lambdas(s.ss_alchemy, 0.0, lam)
    x = s.cartesian()
    q = s.charge
    alpha = s.alphal
    lst = o.alch_listqq(s.ss_alchemy)
    for i, j, _ in lst[:50]:
        a, b = i - 1, j - 1
        r = np.linalg.norm(x[:, a] - x[:, b])
        erfc = oracle.lib().orc_erfc_as(alpha * r)
        t = s.copy()
        sub = oracle.Oracle(t)
        e_add = sub.ferrf_alchemy_add(np.array([[i, j, 1]]), lq)[1].sum()
        total = q[a] * q[b] * erfc / r + (1 - lam) ** 2 * q[a] * q[b] * (1 - erfc) / r + e_add
        assert abs(total - q[a] * q[b] / r) <= 1e-12 * abs(q[a] * q[b] / r)
    f = s.fudge
    for k in range(min(30, len(s.int14))):
        i, j = s.int14[k]
        a, b = i - 1, j - 1
        if abs(s.ss_alchemy[a]) != 2 or abs(s.ss_alchemy[b]) != 2:
            continue
        r = np.linalg.norm(x[:, a] - x[:, b])
        erfc = oracle.lib().orc_erfc_as(alpha * r)
        t = s.copy()
        t.int14 = s.int14[k:k + 1]
        t.type14 = s.type14[k:k + 1]
        e14 = oracle.Oracle(t).fnb14_alchemy(lq, lq)[1][2:].sum()
        recip = (1 - lam) ** 2 * q[a] * q[b] * (1 - erfc) / r
        ferrf = -(1 - f) * (1 - lam) ** 2 * q[a] * q[b] * (1 - erfc) / r
        assert abs(e14 + recip + ferrf - f * q[a] * q[b] / r) <= 1e-12 * abs(q[a] * q[b] / r)
