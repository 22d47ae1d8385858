"""ctypes binding of the in-tree native library (librw.so, include/retainwall.h).

The library is the product: nothing here falls back to Python or to a CPU path.  If
librw.so is missing or cannot be loaded, ``lib()`` raises."""
from __future__ import annotations

import ctypes as ct
import os

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librw.so")

# Every symbol include/retainwall.h declares.
EXPORTS = [
    "rw_status_string", "rw_last_error", "rw_create", "rw_create_from_case", "rw_destroy", "rw_begin_step",
    "rw_neighbor_search", "rw_rigid_body_update", "rw_adami_boundary", "rw_find_corner", "rw_shepard_filter",
    "rw_particle_interaction", "rw_predictor", "rw_corrector", "rw_end_step", "rw_step", "rw_synchronize",
    "rw_wall_force", "rw_save", "rw_get_info", "rw_set_option", "rw_get_array", "rw_set_array", "rw_set_counters",
    "rw_profile", "rw_step_timed", "rw_cell_sort_noalloc", "rw_batch_create", "rw_batch_step",
    "rw_batch_synchronize", "rw_batch_destroy", "rw_batch_wall_force", "rw_autotune", "rw_wall_profile",
    "rw_mlp_last_error", "rw_mlp_create", "rw_mlp_destroy", "rw_mlp_get_params", "rw_mlp_set_params",
    "rw_mlp_forward", "rw_mlp_grad", "rw_mlp_add_samples", "rw_mlp_samples", "rw_mlp_clear_samples",
    "rw_mlp_train", "rw_mlp_feature_ranges", "rw_mlp_collect", "rw_set_closure", "rw_closure_stats",
    "rw_list_stats", "rw_write_case_dat",
]
STAGE_NAMES = ["search_p", "rigid", "adami_p", "corner_p", "interaction_p", "predictor", "search_c", "adami_c",
               "corner_c", "interaction_c", "corrector"]


class RwError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str):
        super().__init__(f"{what}: {_abi.STATUS_NAMES.get(status, status)}: {detail}")
        self.status = status


_lib = None


def lib() -> ct.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not built: run `python -m retainwall_code_b200.build`")
    L = ct.CDLL(LIB_PATH)
    P = ct.c_void_p
    L.rw_status_string.restype = ct.c_char_p
    L.rw_status_string.argtypes = [ct.c_int]
    L.rw_last_error.restype = ct.c_char_p
    L.rw_last_error.argtypes = [P]
    L.rw_create.argtypes = [ct.c_char_p, ct.c_int, ct.c_int, ct.POINTER(P)]
    L.rw_create_from_case.argtypes = [ct.POINTER(_abi.Case), ct.c_int, ct.c_int, ct.POINTER(P)]
    for n in ("rw_destroy", "rw_begin_step", "rw_rigid_body_update", "rw_adami_boundary", "rw_find_corner",
              "rw_shepard_filter", "rw_particle_interaction", "rw_predictor", "rw_corrector", "rw_end_step",
              "rw_synchronize"):
        getattr(L, n).argtypes = [P]
    L.rw_neighbor_search.argtypes = [P, ct.c_int]
    L.rw_step.argtypes = [P, ct.c_int]
    L.rw_step_timed.argtypes = [P, ct.c_int, ct.POINTER(ct.c_double)]
    L.rw_batch_create.argtypes = [ct.POINTER(P), ct.c_int, ct.POINTER(P)]
    L.rw_batch_step.argtypes = [P, ct.c_int, ct.POINTER(ct.c_double)]
    L.rw_batch_synchronize.argtypes = [P]
    L.rw_batch_destroy.argtypes = [P]
    L.rw_batch_wall_force.argtypes = [P, ct.c_int, ct.c_int, ct.c_void_p, ct.POINTER(ct.c_double)]
    L.rw_autotune.argtypes = [P, ct.c_int, ct.POINTER(ct.c_int)]
    L.rw_wall_profile.argtypes = [P, ct.c_double, ct.c_double, ct.c_double, ct.c_int, ct.POINTER(ct.c_double)]
    L.rw_cell_sort_noalloc.argtypes = [ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.rw_wall_force.argtypes = [P, ct.c_int, ct.c_int, ct.c_void_p, ct.POINTER(ct.c_double)]
    L.rw_save.argtypes = [P, ct.c_char_p]
    L.rw_write_case_dat.argtypes = [ct.POINTER(_abi.Case), ct.c_char_p]
    L.rw_get_info.argtypes = [P, ct.POINTER(_abi.Info)]
    L.rw_set_option.argtypes = [P, ct.c_int, ct.c_double]
    L.rw_get_array.argtypes = [P, ct.c_int, ct.c_void_p, ct.c_size_t]
    L.rw_set_array.argtypes = [P, ct.c_int, ct.c_void_p, ct.c_size_t]
    L.rw_set_counters.argtypes = [P, ct.c_double, ct.c_int, ct.c_int, ct.c_int]
    L.rw_profile.argtypes = [P, ct.c_int, ct.POINTER(ct.c_double), ct.c_int, ct.POINTER(ct.c_int)]
    # learned closure
    L.rw_mlp_last_error.restype = ct.c_char_p
    L.rw_mlp_last_error.argtypes = [P]
    L.rw_mlp_create.argtypes = [ct.c_int, ct.c_uint64, ct.c_int64, ct.POINTER(P)]
    L.rw_mlp_destroy.argtypes = [P]
    L.rw_mlp_get_params.argtypes = [P, ct.c_void_p, ct.c_size_t]
    L.rw_mlp_set_params.argtypes = [P, ct.c_void_p, ct.c_size_t]
    L.rw_mlp_forward.argtypes = [P, ct.c_void_p, ct.c_int64, ct.c_void_p]
    L.rw_mlp_grad.argtypes = [P, ct.c_void_p, ct.c_void_p, ct.c_int64, ct.POINTER(ct.c_double), ct.c_void_p]
    L.rw_mlp_add_samples.argtypes = [P, ct.c_void_p, ct.c_void_p, ct.c_int64]
    L.rw_mlp_samples.argtypes = [P, ct.POINTER(ct.c_int64), ct.c_void_p, ct.c_void_p, ct.c_int64]
    L.rw_mlp_clear_samples.argtypes = [P]
    L.rw_mlp_train.argtypes = [P, ct.c_int, ct.c_int, ct.c_float, ct.c_uint64, ct.POINTER(ct.c_double)]
    L.rw_mlp_feature_ranges.argtypes = [P, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.rw_mlp_collect.argtypes = [P, P, ct.c_int, ct.c_void_p, ct.c_uint64, ct.POINTER(ct.c_int64)]
    L.rw_set_closure.argtypes = [P, P, ct.c_double]
    L.rw_closure_stats.argtypes = [P, ct.POINTER(ct.c_double)]
    L.rw_list_stats.argtypes = [P, ct.POINTER(ct.c_int64)]
    _lib = L
    return L


def check(status: int, what: str, ctx=None) -> None:
    if status != 0:
        detail = lib().rw_last_error(ctx)
        raise RwError(status, what, detail.decode() if detail else "")
