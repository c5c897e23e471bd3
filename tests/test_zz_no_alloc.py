"""orac_gpu_pme_kspace_static: the SPME reciprocal sum for callers that
cannot allocate device memory (a host that owns the whole HBM budget, a
serving loop that cannot take the synchronisation cudaMalloc/cudaFree bring,
a plugin forbidden to allocate).  Its scratch is one fixed device array of the
library, so the entry point needs no context and allocates nothing.

The device results are checked against the FP64 oracle's do_pmesh_kspace and
against orac_gpu_do_pmesh_kspace (the context-based entry point) on the same
inputs, on consecutive calls: the array keeps the previous call's contents,
so a call that failed to clear its charge grid or sums would show up on the
second call.  The cases include a 256-point axis (the largest the fixed
scratch takes, 256 x 32 x 32 = 262,144 points in all) and a finite
reciprocal-space cut.  Tolerances are those of the GPU parity tests: forces
relative RMS <= 1e-5, energy relative <= 1e-6, virial <= 1e-5 of its
Frobenius norm.

This file is collected last on purpose; it passes alone in a fresh process
and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from orac_b200 import lib, systems

FORCE_RMS = 1e-5
ENERGY_REL = 1e-6
VIRIAL_REL = 1e-5


def _rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _system():
    s = systems.water_box(nwat=216, box=18.8, lattice=6, jitter=0.25, seeds=(11, 12, 13, 14), nfft=(24, 24, 24))
    s.ncell = None
    return s


def _call(L, stream, n, xyz, q, recip, volume, alpha, order, dims, force, energy, rkcut=0.0):
    err = C.create_string_buffer(512)
    rc = L.orac_gpu_pme_kspace_static(stream, n, xyz.data_ptr(), q.data_ptr(), np.ascontiguousarray(recip.T.ravel()),
                                      volume, alpha, rkcut, order, dims[0], dims[1], dims[2], force.data_ptr(),
                                      energy.data_ptr(), err, len(err))
    return rc, err.value.decode()


def test_capacity_and_argument_errors_without_device_work():
    """Sizes beyond the fixed scratch are rejected before any CUDA call."""
    L = lib.load()
    err = C.create_string_buffer(512)
    recip = np.eye(3) * 0.05
    fake = C.c_void_p(16)  # never dereferenced: the checks come first
    rc = L.orac_gpu_pme_kspace_static(None, 10, fake, fake, recip, 1000.0, 0.35, 0.0, 4, 80, 64, 64, fake, fake,
                                      err, len(err))
    assert rc == 3 and "at most 262144" in err.value.decode(), err.value
    rc = L.orac_gpu_pme_kspace_static(None, 10, fake, fake, recip, 1000.0, 0.35, 0.0, 4, 300, 8, 8, fake, fake,
                                      err, len(err))
    assert rc == 3 and "per axis" in err.value.decode(), err.value
    rc = L.orac_gpu_pme_kspace_static(None, 10, fake, fake, recip, 1000.0, 0.35, 0.0, 6, 4, 8, 8, fake, fake,
                                      err, len(err))
    assert rc == 1 and "fewer than the order" in err.value.decode(), err.value
    rc = L.orac_gpu_pme_kspace_static(None, 10, fake, fake, recip, 1000.0, 0.35, 0.0, 4, 22, 24, 24, fake, fake,
                                      err, len(err))
    assert rc == 1 and "factor" in err.value.decode(), err.value


def _check(F, e, ref, what):
    Fref, eref, vref = ref
    assert _rel_rms(F, Fref) <= FORCE_RMS, f"{what}: force rel RMS {_rel_rms(F, Fref):.3e}"
    assert abs(e[0] - eref) <= ENERGY_REL * abs(eref), f"{what}: eer {e[0]} vs {eref}"
    vir = e[1:].reshape(3, 3, order="F")
    assert np.linalg.norm(vir - vref) <= VIRIAL_REL * np.linalg.norm(vref), f"{what}: virial"


@pytest.mark.gpu
@pytest.mark.parametrize("dims,order,rkcut", [((32, 32, 32), 4, 0.0), ((36, 30, 28), 5, 0.0), ((64, 64, 64), 6, 0.0),
                                              ((256, 32, 32), 4, 0.0), ((32, 32, 32), 4, 1.5)])
def test_static_matches_oracle_and_context_entry_on_consecutive_calls(dims, order, rkcut):
    import torch

    import oracle
    from orac_b200.engine import Engine

    s = _system()
    r = s.cartesian()
    recip = 0.5 * np.linalg.inv(s.co).T
    alpha = 0.35
    refs = {"oracle": oracle.Oracle(s.copy()).do_pmesh_kspace(r[0], r[1], r[2], s.charge, recip, s.volume, alpha,
                                                              order, dims, rkcut if rkcut > 0.0 else 1e9)}
    if rkcut > 0.0:
        # the cut drops modes that matter: the energy moves well beyond the tolerance
        e_full = oracle.Oracle(s.copy()).do_pmesh_kspace(r[0], r[1], r[2], s.charge, recip, s.volume, alpha, order,
                                                         dims)[1]
        assert abs(refs["oracle"][1] - e_full) > 1e-3 * abs(e_full)
    else:
        eng = Engine(s)
        refs["context entry"] = eng.do_pmesh_kspace(r[0], r[1], r[2], s.charge, recip, s.volume, alpha, order, dims)
        eng.close()

    L = lib.load()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    n = s.ntap
    xyz = torch.tensor(np.concatenate([r[0], r[1], r[2]]), dtype=torch.float64, device=dev)
    q = torch.tensor(s.charge, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        force = torch.zeros(3 * n, dtype=torch.float64, device=dev)
        energy = torch.full((10,), float("nan"), dtype=torch.float64, device=dev)
        rc, msg = _call(L, stream, n, xyz, q, recip, s.volume, alpha, order, dims, force, energy, rkcut)
        assert rc == 0, f"call {call}: rc {rc}: {msg}"
        torch.cuda.synchronize(dev)
        F = force.cpu().numpy().reshape(3, n)
        e = energy.cpu().numpy()
        for what, ref in refs.items():
            _check(F, e, ref, f"call {call} vs {what}")

    # forces are accumulated into the caller's array, like the context entry point
    Fref = refs["oracle"][0]
    force = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    energy = torch.zeros(10, dtype=torch.float64, device=dev)
    for _ in range(2):
        rc, msg = _call(L, stream, n, xyz, q, recip, s.volume, alpha, order, dims, force, energy, rkcut)
        assert rc == 0, msg
    torch.cuda.synchronize(dev)
    F2 = force.cpu().numpy().reshape(3, n)
    assert _rel_rms(F2, 2.0 * Fref) <= FORCE_RMS
