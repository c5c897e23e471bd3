"""ctypes binding of liborac_gpu.so (the C ABI declared in include/orac_gpu.h).

The library is built in-tree (orac-porting_b200/Makefile) next to this
module.  Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# ORAC_GPU_LIB selects another in-tree build of the library (tuning sweeps)
LIB_PATH = os.environ.get("ORAC_GPU_LIB") or os.path.join(HERE, "liborac_gpu.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "orac_gpu.h")

ORAC_OK = 0
ERRORS = {1: "ORAC_ERR_PARAM", 2: "ORAC_ERR_CUDA", 3: "ORAC_ERR_CAPACITY", 4: "ORAC_ERR_STATE",
          5: "ORAC_ERR_TIMEOUT", 6: "ORAC_ERR_NODEVICE"}

_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_lib = None


class OracGpuError(RuntimeError):
    pass


def declared_symbols(header=HEADER):
    """Names of every function declared in include/orac_gpu.h."""
    text = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:int|double|const char\s*\*|void\s*\*?)\s*(orac_gpu_\w+)\s*\(", text, re.M)))


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OracGpuError(f"{LIB_PATH} is missing: build it with `make -C orac-porting_b200` (no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    i, d, ch = C.c_int, C.c_double, C.c_char
    i64 = C.c_int64
    sig = {
        "orac_gpu_create": (i, [i, C.POINTER(_P)]),
        "orac_gpu_destroy": (i, [_P]),
        "orac_gpu_last_error": (C.c_char_p, [_P]),
        "orac_gpu_version": (C.c_char_p, []),
        "orac_gpu_set_topology": (i, [_P, i, i, i, _I, _I, _I, _I, _D, _I, i, _I, _D, _D, _D, _D, d, _I, i64]),
        "orac_gpu_set_ewald": (i, [_P, i, d, i, i, i, i, d]),
        "orac_gpu_set_shells": (i, [_P, d, d, d, d, d, d, d, d, d]),
        "orac_gpu_set_linked_cell": (i, [_P, i, i, i]),
        "orac_gpu_set_box": (i, [_P, _D, _D]),
        "orac_gpu_lc_list": (i, [_P, d, _D, _D, _D, C.POINTER(i64)]),
        "orac_gpu_mts_forces": (i, [_P, i, ch, _D, _D, _D, _D, _D, _D, _D, _D, _D, _DP, _DP, _DP, _DP, _DP, _DP,
                                    _DP, _DP, _D, _D, _D, _D]),
        "orac_gpu_fft_pme": (i, [_P, _D, _D, _D, _D, _D, _D, _DP, _D, _D, _D, _D, i]),
        "orac_gpu_do_pmesh_kspace": (i, [_P, i, _D, _D, _D, _D, _D, d, d, i, i, i, i, _DP, _D, _D, _D, _D]),
        "orac_gpu_fnb14": (i, [_P, _D, _D, _D, i, _I, i, _I, _D, _D, i, d, d, _D, _D, _D, _D]),
        "orac_gpu_fnbgrp": (i, [_P, _D, _D, _D, _I, i, _D, _D, _D, _D]),
        "orac_gpu_ferrf": (i, [_P, d, _D, _D, _D, i, _I, i, _D, _D, _D, _D]),
        "orac_gpu_cself": (i, [_P, d, _DP, _DP]),
        "orac_gpu_mts_forces_dev": (i, [_P, ch, _P, _P, _P, _P, _P, _P]),
        "orac_gpu_fft_pme_dev": (i, [_P, _P, _P, _P, _P, _P]),
        "orac_gpu_set_bonded": (i, [_P, i, _I, _D, _D, i, _I, _D, i, _I, _D, _D, i, _I, _D, _D, _D]),
        "orac_gpu_set_intra_pairs": (i, [_P, i, _I, _I, _D, _D, i, d, d, i, _I, i, _I]),
        "orac_gpu_mts_intra_n0": (i, [_P, _D, _D, _D, _D, _D, _D, _D]),
        "orac_gpu_mts_intra_n1": (i, [_P, _D, _D, _D, _D, _D, _D, _D]),
        "orac_gpu_set_rem": (i, [_P, _I, i, d]),
        "orac_gpu_set_alchemy": (i, [_P, _I, _D, _D, d, d, i]),
        "orac_gpu_set_alchemy_shift": (i, [_P, i, d, d]),
        "orac_gpu_set_lambda": (i, [_P, _D, i, i, _P]),
        "orac_gpu_variant_energies": (i, [_P, _D]),
        "orac_gpu_pme_kspace_static": (i, [_P, i, _P, _P, _D, d, d, d, i, i, i, i, _P, _P, C.c_char_p, i]),
        "orac_gpu_md_setup": (i, [_P, _D, _D, _D, _D, _D, _D, _I, _D, i, d, i, i, i, i, i, ch, d]),
        "orac_gpu_md_run": (i, [_P, i, i, _D]),
        "orac_gpu_md_get_state": (i, [_P, _D, _D, _D, _D, _D, _D]),
        "orac_gpu_md_set_graphs": (i, [_P, i]),
        "orac_gpu_md_set_state": (i, [_P, _P, _P, _P, _P, _P, _P]),
        "orac_gpu_md_run_async": (i, [_P, i]),
        "orac_gpu_md_collect": (i, [_P]),
        "orac_gpu_get_stream": (_P, [_P]),
        "orac_gpu_batch_create": (i, [C.POINTER(_P), i, C.POINTER(_P)]),
        "orac_gpu_batch_run": (i, [_P, i]),
        "orac_gpu_batch_run_energy": (i, [_P, i, i]),
        "orac_gpu_batch_set_rem_factors": (i, [_P, _D]),
        "orac_gpu_set_rem_factor_async": (i, [_P, d, _P]),
        "orac_gpu_rem_exchange": (i, [i, _D, _I, _D, d, C.c_longlong, d, _I]),
        "orac_gpu_md_records": (i, [_P, i, _P, C.POINTER(i64), i]),
        "orac_gpu_md_set_schedule": (i, [_P, i, _P, _P, _P, _P, _P, d, i]),
        "orac_gpu_md_work": (i, [_P, _P]),
        "orac_gpu_md_work_trace": (i, [_P, i, _P, C.POINTER(i64)]),
        "orac_gpu_md_set_thermostat": (i, [_P, d, d, d, d]),
        "orac_gpu_md_thermostat": (i, [_P, _P]),
        "orac_gpu_md_set_thermostat_state": (i, [_P, _P, _P]),
        "orac_gpu_batch_sync": (i, [_P]),
        "orac_gpu_batch_destroy": (i, [_P]),
        "orac_gpu_batch_last_error": (C.c_char_p, [_P]),
        "orac_gpu_batch_stream": (_P, [_P]),
        "orac_gpu_counters": (i, [_P, C.POINTER(i64), i]),
        "orac_gpu_prof_enable": (i, [_P, i]),
        "orac_gpu_prof_read": (i, [_P, C.POINTER(d), C.POINTER(i64), i]),
        "orac_gpu_prof_read_family": (i, [_P, i, C.POINTER(d), C.POINTER(i64), i]),
        "orac_gpu_sync": (i, [_P]),
        "orac_gpu_stats": (i, [_P, C.POINTER(i64), C.POINTER(i64)]),
        "orac_gpu_footprint": (i, [_P, C.POINTER(i64)]),
        "orac_gpu_fp32_rate": (i, [i, C.POINTER(d), C.POINTER(d)]),
        "orac_gpu_set_pair_tuning": (i, [_P, i, i, i]),
        "orac_gpu_get_pair_tuning": (i, [_P, C.POINTER(i)]),
        "orac_gpu_tune": (i, [_P, i, C.c_char_p, i, C.POINTER(i), C.POINTER(d)]),
        "orac_gpu_batch_tune": (i, [_P, i, C.c_char_p, i, C.POINTER(i), C.POINTER(d)]),
        "orac_gpu_server_now": (d, []),
        "orac_gpu_server_create": (i, [i, i64, i, i, C.POINTER(_P)]),
        "orac_gpu_server_destroy": (i, [_P]),
        "orac_gpu_server_last_error": (C.c_char_p, [_P]),
        "orac_gpu_server_reserve": (i, [_P, i64, C.POINTER(i)]),
        "orac_gpu_server_unreserve": (i, [_P, i64]),
        "orac_gpu_server_submit": (i, [_P, _P, i, i64, d, C.POINTER(i64)]),
        "orac_gpu_server_poll": (i, [_P, i, _P, _P, _P, _P, C.POINTER(i)]),
        "orac_gpu_server_stats": (i, [_P, C.POINTER(i64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(ctx, rc, what=""):
    if rc != ORAC_OK:
        msg = load().orac_gpu_last_error(ctx).decode() if ctx else ""
        raise OracGpuError(f"{what}: {ERRORS.get(rc, rc)} {msg}")


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def colmajor(m):
    return np.ascontiguousarray(np.asarray(m, dtype=np.float64).T).ravel()
