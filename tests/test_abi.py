"""The C ABI: every entry point include/world_b200.h declares is exported by
libworld_b200.so, and argument errors come back as statuses (no device calls)."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT, gpu_present
from world_b200 import _lib
from world_b200._lib import check, lib

HEADER = os.path.join(ROOT, "include", "world_b200.h")


def declared_symbols() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wd_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_surface():
    names = declared_symbols()
    for required in ("wd_create", "wd_step", "wd_get_state", "wd_set_state",
                     "wd_compute_density_grid", "wd_compute_total_energy", "wd_config_load_yaml"):
        assert required in names
    assert len(names) >= 40


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (wd_[a-z0-9_]+)\b", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for s in declared_symbols():
        assert hasattr(lib, s)
    assert not _lib.MISSING


def test_python_binding_covers_the_header():
    missing = [s for s in declared_symbols() if s not in _lib.SIGNATURES]
    assert not missing, f"no ctypes signature for: {missing}"


def test_null_arguments_are_invalid_not_crashes():
    assert lib.wd_step(None, 1) == -1
    assert "bad argument" in _lib.last_error()
    assert lib.wd_get_state(None, None) == -1
    assert lib.wd_config_create(None) == -1
    assert lib.wd_compute_total_energy(None, None) == -1
    assert lib.wd_destroy(None) == 0


def test_config_get_unknown_key_and_small_buffer():
    cfg = ctypes.c_void_p()
    check(lib.wd_config_create(ctypes.byref(cfg)))
    buf = ctypes.create_string_buffer(64)
    assert lib.wd_config_get(cfg, b"physics", b"nope", buf, 64) == -1
    assert "unknown key" in _lib.last_error()
    tiny = ctypes.create_string_buffer(2)
    assert lib.wd_config_get(cfg, b"initialization", b"type", tiny, 2) == -6
    lib.wd_config_destroy(cfg)


def test_version_string():
    assert b"sm_100a" in lib.wd_version()


@pytest.mark.skipif(gpu_present(), reason="checks the no-device error path")
def test_create_without_a_device_returns_a_cuda_status():
    cfg = ctypes.c_void_p()
    check(lib.wd_config_create(ctypes.byref(cfg)))
    sim = ctypes.c_void_p()
    rc = lib.wd_create(cfg, ctypes.byref(sim))
    assert rc in (-2, -5)
    assert _lib.last_error()
    assert not sim.value
    lib.wd_config_destroy(cfg)


def test_batch_entry_points_take_the_python_argument_forms():
    """The ctypes signatures accept what world_b200.batch passes (numpy buffers via
    ptr(), byref scalars); a NULL handle comes back as WD_ERR_INVALID."""
    import numpy as np
    from world_b200._lib import ptr
    d = np.zeros(8, np.float64)
    i64 = np.zeros(8, np.int64)
    i32 = np.zeros(8, np.int32)
    v = [ctypes.c_int64() for _ in range(4)]
    s = ctypes.c_int32()
    calls = [
        lib.wd_compute_scene_energies(None, ptr(d)),
        lib.wd_compute_scene_momenta(None, ptr(d)),
        lib.wd_scene_overflow_counts(None, ptr(i64)),
        lib.wd_scene_stability(None, ptr(i32)),
        lib.wd_chaos_metrics(None, 0, ptr(d)),
        lib.wd_freeze_scene(None, 0, 1),
        lib.wd_scene_count(None, ctypes.byref(s)),
        lib.wd_scene_range(None, 0, *[ctypes.byref(x) for x in v]),
        lib.wd_create_batch(None, 0, None, None, None, None, None, ctypes.byref(ctypes.c_void_p())),
        lib.wd_set_contact_params(None, 0.5, 0.5, 1e5),
        lib.wd_adjoint_record(None, 10, 5),
        lib.wd_adjoint_backward(None, ptr(d), ptr(d), ptr(d), ptr(d), ptr(d)),
        lib.wd_deposit_vjp(None, ptr(d), ptr(d), ptr(d)),
        lib.wd_write_state_file(None, b"x"),
        lib.wd_write_checkpoint(None, b"x"),
        lib.wd_pack_frame(None, None, ptr(d)),
        lib.wd_set_neighbor_skin(None, 1e-3),
        lib.wd_autotune(None, 10, None, None, None),
        lib.wd_list_stats(None, None, None, None),
        lib.wd_set_state_async(None, ptr(d)),
        lib.wd_get_positions_async(None, ptr(d)),
        lib.wd_io_join(None),
        lib.wd_get_tuning(None, None, None, None),
        lib.wd_set_contact_kernel(None, 256, 0),
        lib.wd_picard_counts(None, None, None),
        lib.wd_list_exact_count(None, None),
    ]
    assert all(c == -1 for c in calls), calls
