"""ctypes binding of libsimp_gpu.so (the C ABI declared in include/simp_gpu.h).

There is no CPU fallback: if the in-tree library is missing, loading fails
with an error that says how to build it.
"""
from __future__ import annotations

import ctypes
import os

from .params import RequestStats, ServerConfig, ServerStats, SimpForcing, SimpParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsimp_gpu.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32

# name -> (restype, argtypes); the symbol list the header declares
SIGNATURES = {
    "simp_params_reference_default": (None, [ctypes.POINTER(SimpParams)]),
    "simp_gpu_create": (_i32, [ctypes.POINTER(SimpParams), _i32, _i32, ctypes.POINTER(_vp)]),
    "simp_gpu_create_batch": (_i32, [ctypes.POINTER(SimpParams), _i32, _i32, _i32, ctypes.POINTER(_vp)]),
    "simp_gpu_destroy": (_i32, [_vp]),
    "simp_gpu_batch_add": (_i32, [_vp, ctypes.POINTER(SimpForcing), _i32, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                  _i32, _dp, _dp, _ip]),
    "simp_gpu_batch_remove": (_i32, [_vp, _i32]),
    "simp_gpu_set_forcing": (_i32, [_vp, ctypes.POINTER(SimpForcing)]),
    "simp_gpu_set_wall_normals": (_i32, [_vp, _i32, _dp]),
    "simp_gpu_batch_get_state": (_i32, [_vp, _i32, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "simp_gpu_batch_info": (_i32, [_vp, _i32, _ip, ctypes.POINTER(ctypes.c_int64), _ip]),
    "simp_gpu_set_state": (_i32, [_vp, _i32, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _i32, _dp, _dp,
                                  ctypes.c_double, ctypes.c_double]),
    "simp_gpu_get_state": (_i32, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "simp_gpu_keep_diag": (_i32, [_vp, _i32]),
    "simp_gpu_get_diag": (_i32, [_vp] + [_dp] * 9),
    "simp_gpu_nnps": (_i32, [_vp, _ip, _ip, _ip, _dp, _dp, _i32, _ip, _ip, _ip, _dp, _i32]),
    "simp_gpu_single_step": (_i32, [_vp, ctypes.c_double, _dp, _dp, _dp, _dp]),
    "simp_gpu_sum_density": (_i32, [_vp, _dp]),
    "simp_gpu_step": (_i32, [_vp, _i32, _dp, _dp]),
    "simp_gpu_interaction_stats": (_i32, [_vp, _ip, _ip, ctypes.POINTER(ctypes.c_int64), _ip]),
    "simp_gpu_sum_density_noalloc": (_i32, [_vp, _vp, _vp, _vp, _i32, _i32, _vp, _vp]),
    "simp_gpu_set_passes": (_i32, [_vp, _i32, _i32, _i32]),
    "simp_gpu_get_passes": (_i32, [_vp, _ip, _ip, _ip]),
    "simp_gpu_autotune": (_i32, [_vp, _i32, _dp]),
    "simp_gpu_stream": (_vp, [_vp]),
    "simp_gpu_kernel_launches": (ctypes.c_int64, [_vp]),
    "simp_gpu_profile": (_i32, [_vp, _i32]),
    "simp_gpu_kernel_times": (_i32, [_vp, _dp, _i32, ctypes.POINTER(ctypes.c_int64)]),
    "simp_gpu_last_error": (ctypes.c_char_p, [_vp]),
    "simp_gpu_version": (ctypes.c_char_p, []),
    # snapshot files (host code; no device needed except for simp_gpu_write_output)
    "simp_csv_create_output": (_i32, [ctypes.c_char_p]),
    "simp_gpu_write_output": (_i32, [_vp, ctypes.c_char_p]),
    "simp_csv_append_snapshot": (_i32, [ctypes.c_char_p, _i32, _i32, ctypes.c_double] + [_dp] * 13),
    "simp_csv_write_walls": (_i32, [ctypes.c_char_p, _i32, _dp, _dp]),
    "simp_csv_read_snapshot": (_i32, [ctypes.c_char_p, _i32, _i32, _ip, _ip, _dp] + [_dp] * 7),
    "simp_csv_read_walls": (_i32, [ctypes.c_char_p, _i32, _ip, _dp, _dp]),
    "simp_csv_last_error": (ctypes.c_char_p, []),
    # include/simp_serve.h
    "simp_server_create": (_i32, [ctypes.POINTER(SimpParams), ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)]),
    "simp_server_destroy": (_i32, [_vp]),
    "simp_server_submit": (_i32, [_vp, ctypes.POINTER(SimpForcing), _i32, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                  _i32, _dp, _dp, ctypes.c_int64, ctypes.c_double, _dp, _dp, _dp, _dp,
                                  ctypes.POINTER(ctypes.c_int64)]),
    "simp_server_run": (_i32, [_vp]),
    "simp_server_cancel": (_i32, [_vp, ctypes.c_int64, ctypes.c_double]),
    "simp_server_request": (_i32, [_vp, ctypes.c_int64, ctypes.POINTER(RequestStats)]),
    "simp_server_stats_get": (_i32, [_vp, ctypes.POINTER(ServerStats)]),
    "simp_server_last_error": (ctypes.c_char_p, [_vp]),
}

_lib = None


class NativeLibraryMissing(ImportError):
    pass


def load(path: str = LIB_PATH):
    """Load the native library (no compute happens at load time)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            f"{path} is not built; run `python -m simp_b200.build` (nvcc, sm_100a). "
            "There is no CPU fallback for the SIMP hot path.")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def iptr(a):
    return None if a is None else a.ctypes.data_as(_ip)
