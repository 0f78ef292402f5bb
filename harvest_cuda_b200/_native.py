"""ctypes binding of the engine's C ABI (``include/harvest_b200.h``).

The shared library is built in-tree by ``harvest_cuda_b200.build``. There is
no CPU fallback: if the library is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes as ct
import os

from . import build as _build

HV_OK = 0
HV_INVALID_ARGUMENT = 1
HV_RUNTIME_ERROR = 2
HV_DEVICE_POINTERS = 1
HV_NO_GRAPH = 2
HV_RECORD_STAGES = 4
HV_NULL_IS_LEGACY_STREAM = 8
HV_STAGE_COUNT = 6

_D = ct.POINTER(ct.c_double)
_L = ct.POINTER(ct.c_int64)

# Every exported entry point with (restype, argtypes); tests check that the
# library exports exactly these and that the header declares them.
SIGNATURES = {
    "hv_last_error": (ct.c_char_p, []),
    "hv_cuda_available": (ct.c_int, [ct.c_int]),
    "hv_output_length": (ct.c_int64, [ct.c_int64, ct.c_int, ct.c_double]),
    "hv_validate": (ct.c_int, [_D, ct.c_int64, ct.c_int, ct.c_double, ct.c_double, ct.c_double]),
    "hv_harvest": (ct.c_int, [_D, ct.c_int64, ct.c_int, ct.c_double, ct.c_double, ct.c_double,
                              ct.c_int, _D, _D, ct.c_int64]),
    "hv_harvest_batch": (ct.c_int, [ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                    ct.c_double, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_uint,
                                    ct.c_void_p]),
    "hv_harvest_batch_pcm16": (ct.c_int, [ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                          ct.c_double, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_uint,
                                          ct.c_void_p]),
    "hv_compare_batch": (ct.c_int, [ct.c_void_p, ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_void_p, ct.c_uint,
                                    ct.c_void_p]),
    "hv_stage_name": (ct.c_char_p, [ct.c_int]),
    "hv_last_stage_ms": (ct.c_int, [_D]),
    "hv_last_tuning": (ct.c_int, [ct.POINTER(ct.c_int)]),
    "hv_profile": (ct.c_int, [_D, ct.c_int64, ct.c_int, ct.c_double, ct.c_double, ct.c_double,
                              ct.c_int, _D, _D, ct.c_int64, _D]),
    "hv_harvest_stages": (ct.c_int, [_D, ct.c_int64, ct.c_int, ct.c_double, ct.c_double, ct.c_int,
                                     _D, _D, ct.POINTER(ct.c_int), _D, _D, _D, _D, _D, _D, _D]),
    "hv_decimate_noalloc": (ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_int, ct.c_void_p,
                                       ct.c_void_p]),
    "hv_harvest_grad_forward": (ct.c_int, [ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                           ct.c_double, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                           ct.c_void_p]),
    "hv_harvest_grad_backward": (ct.c_int, [ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                            ct.c_double, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                            ct.c_void_p]),
    "hv_band_count": (ct.c_int64, [ct.c_double, ct.c_double]),
    "hv_raw_candidates": (ct.c_int, [ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_double, ct.c_double, ct.c_int,
                                     ct.c_void_p, ct.c_void_p]),
    "hv_raw_candidates_backward": (ct.c_int, [ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                              ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "hv_contour_batch": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, _L, ct.c_int, ct.c_int, ct.c_int,
                                    ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_uint, ct.c_void_p]),
    "hv_clear_cache": (ct.c_int, []),
}


def _load():
    path = _build.LIBRARY
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build the CUDA engine first "
            "(python -m harvest_cuda_b200.build); there is no CPU fallback")
    lib = ct.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()
LIBRARY_PATH = _build.LIBRARY


def last_error() -> str:
    msg = lib.hv_last_error()
    return msg.decode() if msg else ""


def raise_for(status: int) -> None:
    """Maps a C-ABI status onto the reference's exception classes."""
    if status == HV_OK:
        return
    message = last_error() or f"harvest failed with status {status}"
    if status == HV_INVALID_ARGUMENT:
        raise ValueError(message)
    raise RuntimeError(message)
