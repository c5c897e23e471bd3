"""Replica exchange on the host (no GPU): the library's decision
(orac_gpu_rem_exchange) against a restatement of ORAC's rem_exchange
(src/rem.f90:371-537) written from the Fortran, and the multi-process
exchange (energies all-gathered, rank 0's random number broadcast) on two
gloo ranks of this machine, which must reach the single-process decision."""
import os
import socket

import numpy as np
import pytest

from orac_b200 import hrem


def orac_rule(ladder, ens, pot, kT, step_rem, random):
    """ORAC's loop as the ranks run it: para_index = ens + 1 (1-based); a
    replica whose mod(step_rem + para_index, 2) != 0 is the low partner of
    para_index + 1 and decides; delta from the ladder and the two
    potentials; accepted: the low replica takes para_index + 1."""
    n = len(ens)
    para = [e + 1 for e in ens]
    new = list(para)
    acc = [0] * (n - 1)
    for r in range(n):
        p = para[r]
        if (step_rem + p) % 2 != 0 and p != n:
            hi = para.index(p + 1)
            delta = (ladder[p] - ladder[p - 1]) * (pot[hi] - pot[r]) / kT
            if delta >= 0.0 or random <= np.exp(delta):
                new[r], new[hi] = p + 1, p
                acc[p - 1] = 1
    return np.array(new) - 1, np.array(acc)


@pytest.mark.parametrize("seed", range(6))
def test_decision_is_orac_rule(seed):
    rng = np.random.default_rng(seed)
    n = 7
    ladder = hrem.ladder_geometric(n, 0.4)
    ens = rng.permutation(n).astype(np.int32)
    pot = rng.normal(-50.0, 20.0, n)
    for step in range(4):
        r = rng.random()
        got, acc = hrem.decide(ladder, ens, pot, 2.5, step, r)
        want, wacc = orac_rule(ladder, list(ens), pot, 2.5, step, r)
        assert np.array_equal(got, want) and np.array_equal(acc, wacc)
        assert sorted(got) == list(range(n))
        ens = got


def test_decision_rejects_a_non_permutation():
    from orac_b200 import lib

    with pytest.raises(lib.OracGpuError):
        hrem.decide(np.ones(3), np.array([0, 0, 1]), np.zeros(3), 1.0, 0, 0.5)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, ws, port, pot_all, ladder, ens, kT, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        n = len(pot_all)
        lo, hi = rank * n // ws, (rank + 1) * n // ws
        rng = np.random.default_rng(123)
        out = []
        e = np.array(ens, dtype=np.int32)
        for step in range(3):
            e, acc = hrem.exchange_distributed(pot_all[lo:hi] + step, e, ladder, kT, step, rng=rng)
            out.append((e.tolist(), acc.tolist()))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_exchange_across_two_ranks_matches_one_process():
    import multiprocessing as mp

    n, ws = 6, 2
    rng = np.random.default_rng(5)
    pot = rng.normal(-30.0, 15.0, n)
    ladder = hrem.ladder_geometric(n, 0.5)
    ens = list(range(n))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, pot, ladder, ens, 1.7, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1]
    # the same rounds in one process, rank 0's random numbers
    r0 = np.random.default_rng(123)
    e = np.array(ens, dtype=np.int32)
    for step in range(3):
        e, acc = hrem.decide(ladder, e, pot + step, 1.7, step, r0.random())
        assert res[0][step] == (e.tolist(), acc.tolist())
