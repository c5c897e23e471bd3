"""The C ABI library without a GPU: it loads, exports every entry point its
header declares, and reports the absence of a device as a status code."""
import ctypes as C
import os

import pytest

from orac_b200 import lib


def test_library_exports_every_declared_symbol():
    L = lib.load()
    names = lib.declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_header_cites_reference_routines():
    text = open(lib.HEADER).read()
    for ref in ("src/mts_forces.f", "src/lc_list.f", "src/fft_pme.f", "src/pme_fftw3.f90", "src/fnb14.f",
                "src/fnbgrp.f", "src/ferrf.f", "src/cself.f"):
        assert ref in text


def test_version_string():
    assert b"sm_100a" in lib.load().orac_gpu_version()


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device status")
def test_create_without_device_returns_status():
    ctx = C.c_void_p()
    rc = lib.load().orac_gpu_create(0, C.byref(ctx))
    assert rc == 6  # ORAC_ERR_NODEVICE
    assert not ctx.value


def test_errors_before_setup_are_status_codes():
    L = lib.load()
    # a null context is rejected without touching the device
    assert L.orac_gpu_destroy(None) == 0
    assert L.orac_gpu_sync(None) == 1
