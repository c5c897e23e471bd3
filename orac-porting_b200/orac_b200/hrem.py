"""Hamiltonian replica exchange: ORAC's HREM (src/rem.f90) for replicas of
one system that differ in the scaling of a solute segment (rem_factor(3)
on the segment's nonbonded pairs, force_rem).

ORAC runs one replica per MPI rank and, every exchange interval, lets
neighbouring ensembles of the scaling ladder trade places by a Metropolis
test on the replicas' segment energies (rem_exchange,
src/rem.f90:371-537): the ensemble index moves, the coordinates stay.  Here
the replicas of one GPU are the members of a Batch (one graph launch per
step advances all of them); every exchange interval ends with an energy
step whose record (column 15, written on the device) holds each replica's
segment energy; the decision is the library's orac_gpu_rem_exchange; an
accepted swap rewrites the two replicas' rem_factor on the device
(orac_gpu_batch_set_rem_factors), so no step graph is captured again.

Across GPUs (one process per GPU, each holding a contiguous block of the
replicas), the segment energies are all-gathered over torch.distributed and
rank 0's random number is broadcast, as ORAC's MPI_ALLGATHER / MPI_BCAST do
(src/rem.f90:286-295, 428-451); every rank then reaches the same decision
and applies it to its own replicas.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as L


def ladder_geometric(n, smin):
    """n scaling factors from 1 down to smin, geometric (ORAC's REM.set of
    test2: 1, 0.843, 0.711, 0.6 for four replicas down to 0.6)."""
    if n == 1:
        return np.ones(1)
    return smin ** (np.arange(n) / (n - 1))


def decide(ladder, ens, pot, kT, step_rem, random):
    """ORAC's exchange decision (orac_gpu_rem_exchange): the new ensemble of
    every replica and, per ensemble pair (p, p + 1), whether it swapped."""
    lib = L.load()
    n = len(ens)
    e = np.ascontiguousarray(ens, dtype=np.int32).copy()
    acc = np.zeros(max(1, n - 1), np.int32)
    rc = lib.orac_gpu_rem_exchange(n, np.ascontiguousarray(ladder, dtype=np.float64), e,
                                   np.ascontiguousarray(pot, dtype=np.float64), float(kT), int(step_rem), float(random),
                                   acc)
    if rc != L.ORAC_OK:
        raise L.OracGpuError(f"orac_gpu_rem_exchange: {L.ERRORS.get(rc, rc)}")
    return e, acc[:n - 1]


class HremBatch:
    """Replicas of one system batched on one GPU with exchanges every
    `every` steps.  engines[r] must carry orac_gpu_set_rem with the ladder's
    segment and be set up for MD; replica r starts in ensemble r."""

    def __init__(self, engines, ladder, kT, seed=0):
        from .engine import Batch

        self.engines = list(engines)
        self.ladder = np.asarray(ladder, dtype=np.float64)
        self.kT = float(kT)
        self.rng = np.random.default_rng(seed)
        self.ens = np.arange(len(self.engines), dtype=np.int32)
        self.step_rem = 0
        self.attempts = np.zeros(max(1, len(self.engines) - 1), np.int64)
        self.accepts = np.zeros(max(1, len(self.engines) - 1), np.int64)
        self.batch = Batch(self.engines)
        self.batch.set_rem_factors(self.ladder[self.ens])

    def segment_energies(self):
        return np.array([e.md_records(1)[0][-1, 15] for e in self.engines])

    def interval(self, every):
        """`every` batched steps, the last an energy step, then one exchange."""
        self.batch.run(every, sync=True, energy_every=every)
        pot = self.segment_energies()
        self.step_rem += 1
        random = self.rng.random()
        for p in range(len(self.engines) - 1):
            if (self.step_rem + p + 1) % 2 == 1:
                self.attempts[p] += 1
        self.ens, acc = decide(self.ladder, self.ens, pot, self.kT, self.step_rem, random)
        self.accepts[:len(acc)] += acc
        self.batch.set_rem_factors(self.ladder[self.ens])
        return pot

    def acceptance(self):
        return np.where(self.attempts > 0, self.accepts / np.maximum(self.attempts, 1), 0.0)

    def close(self):
        self.batch.close()


def exchange_distributed(local_pot, ens_global, ladder, kT, step_rem, rng=None, group=None, device=None):
    """One exchange across ranks: every rank holds a contiguous block of the
    replicas (local_pot, its replicas' segment energies); the energies are
    all-gathered, rank 0's random number broadcast, and every rank returns
    the same new ensemble of every replica and the pairs that swapped."""
    import torch
    import torch.distributed as dist

    dev = torch.device("cpu") if device is None else device
    ws = dist.get_world_size(group)
    mine = torch.tensor(np.asarray(local_pot, dtype=np.float64), device=dev)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(ws)]
    dist.all_gather(sizes, torch.tensor([mine.numel()], dtype=torch.int64, device=dev), group=group)
    nmax = int(max(int(x.item()) for x in sizes))
    pad = torch.zeros(nmax, dtype=torch.float64, device=dev)
    pad[:mine.numel()] = mine
    parts = [torch.zeros(nmax, dtype=torch.float64, device=dev) for _ in range(ws)]
    dist.all_gather(parts, pad, group=group)
    pot = np.concatenate([parts[r][:int(sizes[r].item())].cpu().numpy() for r in range(ws)])
    rnd = torch.zeros(1, dtype=torch.float64, device=dev)
    if dist.get_rank(group) == 0:
        rnd[0] = (rng or np.random.default_rng()).random()
    dist.broadcast(rnd, src=0, group=group)
    return decide(ladder, ens_global, pot, kT, step_rem, float(rnd.item()))
