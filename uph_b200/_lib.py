"""Loads libuph.so (the in-tree CUDA build) and declares its C ABI.

There is no CPU fallback: if the library is missing the import of
uph_b200.sim fails with the build command to run.
"""
from __future__ import annotations

import ctypes as C
import os

from ._capi import SurConfig, SurJudge, SurNodes, SurReport, UphDiagnostics, UphParams, UphStats

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libuph.so")
LIB_SPH_PATH = os.path.join(HERE, "libuph_sph.so")
LIB_DRIVER_PATH = os.path.join(HERE, "libuph_driver.so")

_lib = None

# every exported symbol of include/uph.h with (restype, argtypes)
SIGNATURES = {
    "uph_params_from_file": (C.c_int, [C.c_char_p, C.c_double, C.POINTER(UphParams)]),
    "uph_params_derive": (C.c_int, [C.POINTER(UphParams), C.c_double]),
    "uph_deck_read": (C.c_int, [C.c_char_p, C.c_double, C.POINTER(UphParams), C.c_void_p]),
    "uph_sim_create": (C.c_int, [C.POINTER(UphParams), C.POINTER(C.c_void_p)]),
    "uph_sim_destroy": (C.c_int, [C.c_void_p]),
    "uph_sim_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "uph_sim_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "uph_sim_download": (C.c_int, [C.c_void_p, C.c_void_p]),
    "uph_sim_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "uph_sim_set_graph": (C.c_int, [C.c_void_p, C.c_int32]),
    "uph_sim_set_fused_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "uph_sim_set_candidate_lists": (C.c_int, [C.c_void_p, C.c_int32]),
    "uph_sim_set_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "uph_sim_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32 * 3), C.POINTER(C.c_double)]),
    "uph_sim_set_wall_motion": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "uph_sim_set_wall_base": (C.c_int, [C.c_void_p, C.c_void_p]),
    "uph_sim_derivatives": (C.c_int, [C.c_void_p, C.c_double]),
    "uph_sim_pairs": (C.c_int, [C.c_void_p, C.c_int64] + [C.c_void_p] * 5 + [C.POINTER(C.c_int64)]),
    "uph_sim_stats": (C.c_int, [C.c_void_p, C.POINTER(UphStats)]),
    "uph_sim_approx_vorticity": (C.c_int, [C.c_void_p, C.c_void_p]),
    "uph_sim_virtual": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(C.c_int64)]),
    "uph_sim_set_diagnostics": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double]),
    "uph_sim_diagnostics": (C.c_int, [C.c_void_p, C.POINTER(UphDiagnostics)]),
    "uph_write_output": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(UphParams), C.c_void_p, C.c_void_p,
                                   C.POINTER(UphDiagnostics)]),
    "uph_sim_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "uph_sim_kernel_times": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t,
                                       C.POINTER(C.c_int32)]),
    "uph_sim_launch_count": (C.c_int64, [C.c_void_p]),
    "uph_search_neighbors": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                       C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]),
    "uph_search_neighbors_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                               C.POINTER(C.c_double * 2), C.POINTER(C.c_double * 2), C.c_int64,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64),
                                               C.c_void_p]),
    "uph_rcp_selftest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    # include/uph_surrogate.h
    "uph_tc_gemm_bf16": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                   C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                   C.c_int32, C.c_void_p, C.c_void_p]),
    "uph_tc_wait_selftest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "uph_sur_create": (C.c_int, [C.POINTER(SurConfig), C.c_int32, C.POINTER(C.c_void_p)]),
    "uph_sur_destroy": (C.c_int, [C.c_void_p]),
    "uph_sur_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "uph_sur_param_count": (C.c_int64, [C.c_int32]),
    "uph_sur_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "uph_sur_get_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "uph_sur_reset_optimizer": (C.c_int, [C.c_void_p]),
    "uph_sur_set_fused": (C.c_int, [C.c_void_p, C.c_int32]),
    "uph_sur_forward": (C.c_int, [C.c_void_p, C.POINTER(SurNodes), C.c_void_p]),
    "uph_sur_gradients": (C.c_int, [C.c_void_p, C.POINTER(SurNodes), C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_double)]),
    "uph_sur_adam": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
    "uph_sur_advance": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(SurJudge), C.POINTER(SurReport)]),
    "uph_status_string": (C.c_char_p, [C.c_int]),
    "uph_last_error": (C.c_char_p, []),
}


class UphError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        name = lib().uph_status_string(status).decode()
        super().__init__(f"{where}: {name}: {message}")
        self.status_name = name


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m uph_b200.build` "
                              "(the GPU path has no CPU fallback)")
        l = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def check(status: int, where: str) -> None:
    if status != 0:
        raise UphError(status, where, lib().uph_last_error().decode())
