"""ctypes binding of libworld_b200.so (declarations: include/world_b200.h).

The library is the product: there is no Python or CPU fallback. Importing this
module without the built library raises at once.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_uint8, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("WORLD_B200_LIB", os.path.join(HERE, "libworld_b200.so"))

WD_OK = 0
WD_WARN_DEFAULTS = 1
WD_WARN_UNKNOWN_KEY = 2
WD_HIST_CAP = 24
WD_NOALLOC_MAX_NODES = 64 * 64 * 64

_STATUS_NAMES = {
    -1: "WD_ERR_INVALID", -2: "WD_ERR_CUDA", -3: "WD_ERR_IO", -4: "WD_ERR_CONFIG",
    -5: "WD_ERR_OOM", -6: "WD_ERR_CAPACITY",
}


class WorldError(RuntimeError):
    """A libworld_b200 call returned an error status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libworld_b200.so not found at {LIB_PATH}; build it with "
            "`python world_b200/build.py` (nvcc, sm_100a)")
    return ctypes.CDLL(LIB_PATH)


lib = _load()

_f = POINTER(c_float)
_i32 = POINTER(c_int32)
_i64 = POINTER(c_int64)
_d = POINTER(c_double)
_u8 = POINTER(c_uint8)
_p = c_void_p

SIGNATURES = {
    "wd_last_error": ([], c_char_p),
    "wd_version": ([], c_char_p),
    "wd_config_create": ([POINTER(c_void_p)], c_int),
    "wd_config_destroy": ([_p], c_int),
    "wd_config_copy": ([_p, POINTER(c_void_p)], c_int),
    "wd_config_load_yaml": ([_p, c_char_p], c_int),
    "wd_config_set": ([_p, c_char_p, c_char_p, c_char_p], c_int),
    "wd_config_get": ([_p, c_char_p, c_char_p, c_char_p, c_size_t], c_int),
    "wd_initial_state": ([_p, _p, _p, c_int64, _i64], c_int),
    "wd_create": ([_p, POINTER(c_void_p)], c_int),
    "wd_create_from_arrays": ([_p, c_int64, _p, _p, _p, _p, POINTER(c_void_p)], c_int),
    "wd_create_batch": ([_p, c_int32, _p, _p, _p, _p, _p, POINTER(c_void_p)], c_int),
    "wd_scene_count": ([_p, POINTER(c_int32)], c_int),
    "wd_scene_range": ([_p, c_int32, _i64, _i64, _i64, _i64], c_int),
    "wd_compute_scene_energies": ([_p, _p], c_int),
    "wd_compute_scene_momenta": ([_p, _p], c_int),
    "wd_scene_overflow_counts": ([_p, _p], c_int),
    "wd_scene_stability": ([_p, _p], c_int),
    "wd_freeze_scene": ([_p, c_int32, c_int32], c_int),
    "wd_chaos_metrics": ([_p, c_int32, _p], c_int),
    "wd_write_state_file": ([_p, c_char_p], c_int),
    "wd_write_checkpoint": ([_p, c_char_p], c_int),
    "wd_create_from_checkpoint": ([_p, c_char_p, POINTER(c_void_p)], c_int),
    "wd_pack_frame": ([_p, _p, _p], c_int),
    "wd_list_stats": ([_p, _i64, POINTER(c_int32), _d], c_int),
    "wd_set_neighbor_skin": ([_p, c_float], c_int),
    "wd_picard_counts": ([_p, _i64, _i64], c_int),
    "wd_list_exact_count": ([_p, _i64], c_int),
    "wd_list_resort_count": ([_p, _i64], c_int),
    "wd_get_tuning": ([_p, POINTER(c_float), POINTER(c_int32), POINTER(c_int32)], c_int),
    "wd_set_contact_kernel": ([_p, c_int32, c_int32], c_int),
    "wd_set_build_kernel": ([_p, c_int32], c_int),
    "wd_debug_stage_wait": ([_p, c_int32, c_int32], c_int),
    "wd_set_state_async": ([_p, _p], c_int),
    "wd_get_positions_async": ([_p, _p], c_int),
    "wd_io_join": ([_p], c_int),
    "wd_autotune": ([_p, c_int32, c_char_p, POINTER(c_float), POINTER(c_int32)], c_int),
    "wd_set_contact_params": ([_p, c_float, c_float, c_float], c_int),
    "wd_adjoint_record": ([_p, c_int64, c_int32], c_int),
    "wd_adjoint_backward": ([_p, _p, _p, _p, _p, _p], c_int),
    "wd_deposit_vjp": ([_p, _p, _p, _p], c_int),
    "wd_destroy": ([_p], c_int),
    "wd_step": ([_p, c_int64], c_int),
    "wd_set_dt": ([_p, c_float], c_int),
    "wd_get_dt": ([_p, _f], c_int),
    "wd_get_time": ([_p, _f], c_int),
    "wd_set_time": ([_p, c_float], c_int),
    "wd_get_n": ([_p, _i64], c_int),
    "wd_get_picard_stats": ([_p, _i32, _f], c_int),
    "wd_set_state": ([_p, _p], c_int),
    "wd_get_state": ([_p, _p], c_int),
    "wd_get_positions": ([_p, _p], c_int),
    "wd_get_rhs": ([_p, _p], c_int),
    "wd_get_grain_props": ([_p, _p, _p, _p], c_int),
    "wd_set_state_device": ([_p, _p], c_int),
    "wd_get_state_device": ([_p, _p], c_int),
    "wd_get_positions_device": ([_p, _p], c_int),
    "wd_set_stream": ([_p, _p], c_int),
    "wd_get_stream": ([_p, POINTER(c_void_p)], c_int),
    "wd_synchronize": ([_p], c_int),
    "wd_get_history": ([_p, _p, _p, _p], c_int),
    "wd_set_history": ([_p, _p, _p, _p], c_int),
    "wd_density_grid_nodes": ([_p, _i64], c_int),
    "wd_compute_density_grid": ([_p, _p], c_int),
    "wd_compute_density_grid_device": ([_p, _p], c_int),
    "wd_compute_total_energy": ([_p, _d], c_int),
    "wd_grain_energies": ([_p, _p], c_int),
    "wd_compute_momentum": ([_p, _d], c_int),
    "wd_is_stable": ([_p, _i32], c_int),
    "wd_compute_max_acceleration": ([_p, _f], c_int),
    "wd_grid_overflow_count": ([_p, _i64], c_int),
    "wd_history_overflow_count": ([_p, _i64], c_int),
    "wd_timings": ([_p, _f], c_int),
    "wd_set_kernel_timing": ([_p, c_int32], c_int),
    "wd_radix_search_count": ([_p, _i64, _i32], c_int),
    "wd_kernels_per_step": ([_p, _i64], c_int),
    "wd_deposit_grid_noalloc": ([_p, _p, c_int64, _p, _p, _p, _p, _p], c_int),
    "wd_debug_cell_keys": ([_p, _p], c_int),
    "wd_debug_sorted": ([_p, _p, _p], c_int),
    "wd_debug_candidates": ([_p, _p, _p, _p, c_int64, _i64], c_int),
}

# A library built before an entry point existed loads too; calling that entry point
# then raises AttributeError (tests/test_abi.py checks that the built library exports
# every declared symbol).
MISSING = []
for _name, (_args, _res) in SIGNATURES.items():
    try:
        _fn = getattr(lib, _name)
    except AttributeError:
        MISSING.append(_name)
        continue
    _fn.argtypes = _args
    _fn.restype = _res


def last_error() -> str:
    return lib.wd_last_error().decode("utf-8", "replace")


def check(status: int) -> int:
    """Raise WorldError for negative statuses; return warnings (> 0) unchanged."""
    if status < 0:
        raise WorldError(status, last_error())
    return status


def ptr(array) -> c_void_p:
    """Address of a numpy array's buffer (must be contiguous) or a torch tensor's data."""
    if array is None:
        return c_void_p(None)
    if hasattr(array, "data_ptr"):
        return c_void_p(array.data_ptr())
    if not array.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return c_void_p(array.ctypes.data)
