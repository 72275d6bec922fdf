"""The allocation-free CIC deposit, wd_deposit_grid_noalloc.

It exists for callers that cannot call cudaMalloc: processes whose device memory
belongs to another framework's allocator, and loops that must not allocate while
they run. It takes the caller's own device arrays and keeps its scratch in one
static device array, so it has to give the same field as the allocating entry
point (wd_compute_density_grid) and must not carry anything over from one call to
the next. This file is collected last on purpose: if it fails, a run that stops at
the first failure has already run everything else.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from world_b200 import ParticleDynamics, SimConfig
from world_b200._lib import WD_NOALLOC_MAX_NODES, lib, ptr

pytestmark = pytest.mark.gpu


def _grid_args(cfg):
    lo = (ctypes.c_float * 3)(cfg.domain.x_min, cfg.domain.y_min, cfg.domain.z_min)
    hi = (ctypes.c_float * 3)(cfg.domain.x_max, cfg.domain.y_max, cfg.domain.z_max)
    size = (ctypes.c_int32 * 3)(cfg.density_grid_size_x, cfg.density_grid_size_y,
                                cfg.density_grid_size_z)
    return lo, hi, size


def test_matches_allocating_deposit_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    cfg = SimConfig()
    cfg.init_jitter = 0.3
    cfg.init_vx0, cfg.init_vy0, cfg.init_vz0 = 0.5, -0.25, 0.1   # all channels non-zero
    cfg.kernel_timing = False
    sim = ParticleDynamics(cfg)
    nodes = sim.density_grid_nodes()
    assert nodes <= WD_NOALLOC_MAX_NODES
    mass = torch.from_numpy(sim.grain_mass.copy()).cuda()
    lo, hi, size = _grid_args(cfg)
    for call in range(2):
        state = sim.state_tensor()
        out = torch.full((4 * nodes,), float("nan"), dtype=torch.float32, device="cuda")
        rc = lib.wd_deposit_grid_noalloc(ptr(state), ptr(mass), sim.n, lo, hi, size, ptr(out), None)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(4, -1)
        sim.compute_density_grid()
        want = sim.host_density_grid.reshape(4, -1)
        for c in range(4):
            assert np.abs(want[c]).max() > 0
        # same float products, same per-channel scale, integer sums: the same bits
        np.testing.assert_array_equal(got, want, err_msg=f"call {call}")
        # the state moves between the two calls, so stale sums would show
        sim.advance(40)
    # no grains: an all-zero field that still overwrites the caller's buffer
    out = torch.full((4 * nodes,), float("nan"), dtype=torch.float32, device="cuda")
    assert lib.wd_deposit_grid_noalloc(None, None, 0, lo, hi, size, ptr(out), None) == 0
    torch.cuda.synchronize()
    assert not out.any().item() and not out.isnan().any().item()
    sim.close()


def test_non_finite_momentum_gives_a_nan_channel():
    torch = pytest.importorskip("torch")
    cfg = SimConfig()
    cfg.init_jitter = 0.3
    cfg.kernel_timing = False
    sim = ParticleDynamics(cfg)
    nodes = sim.density_grid_nodes()
    state = sim.state_tensor().clone().reshape(-1, 6)
    state[7, 4] = float("inf")            # one grain's vy
    mass = torch.from_numpy(sim.grain_mass.copy()).cuda()
    lo, hi, size = _grid_args(cfg)
    out = torch.zeros(4 * nodes, dtype=torch.float32, device="cuda")
    assert lib.wd_deposit_grid_noalloc(ptr(state), ptr(mass), sim.n, lo, hi, size, ptr(out),
                                       None) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(4, -1)
    assert np.isnan(got[2]).all()
    assert np.isfinite(got[[0, 1, 3]]).all() and got[0].sum() > 0
    sim.close()


def test_grid_above_the_fixed_scratch_is_rejected():
    lo = (ctypes.c_float * 3)(-1, -1, -1)
    hi = (ctypes.c_float * 3)(1, 1, 1)
    size = (ctypes.c_int32 * 3)(65, 64, 64)
    out = ctypes.c_void_p(1)    # never touched: the size check comes first
    rc = lib.wd_deposit_grid_noalloc(None, None, 0, lo, hi, size, out, None)
    assert rc == -6
    assert "exceeds" in lib.wd_last_error().decode()
