"""The ParticleDynamics / C-ABI surface on the GPU: state in and out, dt changes,
graph and timed launch paths, checkpoint / resume of the tangential history,
PyTorch zero-copy, diagnostics and their error paths."""
from __future__ import annotations

import ctypes

import os

import numpy as np
import pytest

from world_b200 import ParticleDynamics, SimConfig, WorldError
from world_b200._lib import check, lib, ptr
from world_b200.state_io import initial_state

pytestmark = pytest.mark.gpu


def jitter_cfg(**kw):
    cfg = SimConfig()
    cfg.init_jitter = 0.3
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def test_state_round_trip_and_positions():
    sim = ParticleDynamics(jitter_cfg())
    rng = np.random.default_rng(0)
    st = sim.get_state().reshape(-1, 6)
    st[:, 3:] = rng.normal(0, 0.1, (sim.n, 3)).astype(np.float32)
    sim.set_state(st)
    assert np.array_equal(sim.get_state(), st.reshape(-1))
    assert np.array_equal(sim.get_positions(), st[:, :3].reshape(-1))
    sim.advance(10)
    st2 = sim.get_state()
    sim.set_state(st2)                  # set after the order has been permuted
    assert np.array_equal(sim.get_state(), st2)


def test_graph_and_timed_paths_are_identical():
    a = ParticleDynamics(jitter_cfg(kernel_timing=True))
    b = ParticleDynamics(jitter_cfg(kernel_timing=False))
    a.advance(120)
    b.advance(120)
    assert np.array_equal(a.get_state(), b.get_state())
    t = a._timings()
    assert t[0] > 0 and t[1] > 0


def test_dt_change_applies_to_next_step(oracle_for):
    cfg = jitter_cfg(kernel_timing=False)
    st, _ = initial_state(cfg)
    sim = ParticleDynamics(cfg)
    orc = oracle_for(cfg, st)
    sim.advance(20)
    orc.step(20)
    sim.dt = 5e-5
    orc.p.dt = np.float32(5e-5)
    sim.advance(20)
    orc.step(20)
    assert np.array_equal(sim.get_state(), orc.state)
    assert sim.time == pytest.approx(20 * 1e-4 + 20 * 5e-5, rel=1e-5)


def test_history_checkpoint_resume_is_bit_identical():
    cfg = jitter_cfg(history=True, kernel_timing=False)
    a = ParticleDynamics(cfg)
    a.advance(60)
    state = a.get_state()
    hist = a.get_history()
    assert hist[0].sum() > 0
    a.advance(60)
    b = ParticleDynamics(cfg)
    b.set_state(state)
    b.set_history(*hist)
    b.advance(60)
    assert np.array_equal(a.get_state(), b.get_state())


def test_set_history_needs_history_mode():
    sim = ParticleDynamics(jitter_cfg())
    cnt, part, xi = sim.get_history()
    assert cnt.sum() == 0
    with pytest.raises(WorldError):
        sim.set_history(cnt, part, xi)


def test_torch_zero_copy_and_external_stream():
    torch = pytest.importorskip("torch")
    sim = ParticleDynamics(jitter_cfg(kernel_timing=False))
    t = sim.state_tensor()
    assert np.array_equal(t.cpu().numpy(), sim.get_state())
    t[3::6] += 0.25
    sim.set_state_tensor(t)
    assert np.array_equal(sim.get_state(), t.cpu().numpy())
    s = torch.cuda.Stream()
    check(lib.wd_set_stream(sim.handle, ctypes.c_void_p(s.cuda_stream)))
    ref = ParticleDynamics(jitter_cfg(kernel_timing=False))
    ref.set_state(t.cpu().numpy())
    sim.advance(30)
    ref.advance(30)
    assert np.array_equal(sim.get_state(), ref.get_state())
    check(lib.wd_set_stream(sim.handle, None))
    dev = torch.empty(3 * sim.n, dtype=torch.float32, device="cuda")
    check(lib.wd_get_positions_device(sim.handle, ptr(dev)))
    sim.synchronize()
    assert np.array_equal(dev.cpu().numpy(), sim.get_positions())


def test_is_stable_detects_escape_and_nan():
    sim = ParticleDynamics()
    assert sim.is_stable()
    st = sim.get_state()
    st[0] = 5.0
    sim.set_state(st)
    assert not sim.is_stable()
    st[0] = np.nan
    sim.set_state(st)
    assert not sim.is_stable()


def test_max_acceleration_matches_rhs():
    sim = ParticleDynamics(jitter_cfg())
    sim.advance(50)
    a = sim.get_rhs().reshape(-1, 6)[:, 3:]
    sq = (a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1]).astype(np.float32) + a[:, 2] * a[:, 2]
    assert sim.compute_max_acceleration() == np.sqrt(sq.astype(np.float32)).max()


def test_picard_stats_and_launch_count():
    cfg = jitter_cfg(time_integrator="backward_euler_picard", picard_iterations=6,
                     picard_tolerance=1e-7, kernel_timing=False)
    sim = ParticleDynamics(cfg)
    sim.advance(5)
    used, res = sim.picard_stats()
    assert 1 <= used < 6 and res < 1e-7
    # per iteration on the incremental path: keys, mover kernel, merge, gather,
    # contact; a search on the radix path adds by-id + 3 kernels per pass
    # (32^3 cells -> 15-bit keys -> 2 passes of 8 bits)
    assert sim.kernels_per_step() == 6 * 5
    radix, each = sim.radix_search_count()
    assert radix == 0 and each == 1 + 3 * 2      # 1000 grains always fit the mover path
    big = SimConfig()
    big.cube_length_x = big.cube_length_y = big.cube_length_z = 0.65   # 32^3 grains
    big.init_jitter = 0.25
    big.kernel_timing = False
    sim = ParticleDynamics(big)
    sim.advance(3)
    radix, _ = sim.radix_search_count()
    assert radix == 1        # only the first search (every grain is new) sorts them all


def test_create_errors_are_statuses(tmp_path):
    cfg = SimConfig()
    cfg.init_type = "file"
    cfg.init_state_path = str(tmp_path / "missing.bin")
    with pytest.raises(WorldError) as e:
        ParticleDynamics(cfg)
    assert e.value.status == -3
    cfg = SimConfig()
    cfg.particle_material = 7          # no such entry in materials.masses
    with pytest.raises(WorldError):
        ParticleDynamics(cfg)
    with pytest.raises(ValueError):
        ParticleDynamics(SimConfig(), state=np.zeros((4, 6), np.float32), radius=np.ones(3, np.float32))


def test_checkpoint_resume_is_bit_identical(tmp_path):
    from test_gpu_parity import packed_poly
    from world_b200.state_io import read_checkpoint, read_state_file
    cfg, st, rad = packed_poly(n=1500, seed=31, mu=0.5)
    a = ParticleDynamics(cfg, state=st, radius=rad)
    a.advance(60)
    a.dt = 8e-6                      # the checkpoint carries dt too
    a.advance(5)
    path = str(tmp_path / "ck.bin")
    a.write_checkpoint(path)
    ck = read_checkpoint(path, verify=True)
    assert not os.path.exists(path + ".tmp") and not os.path.exists(path + ".sidecar.tmp")
    np.testing.assert_array_equal(ck["state"].reshape(-1), a.get_state())
    assert ck["time"] == np.float32(a.time) and ck["dt"] == np.float32(8e-6)
    cnt, part, xi = a.get_history()
    np.testing.assert_array_equal(ck["count"], cnt)
    assert cnt.sum() > 0
    a.advance(40)
    b = ParticleDynamics.from_checkpoint(cfg, path)
    assert b.time == ck["time"]
    b.advance(40)
    np.testing.assert_array_equal(b.get_state(), a.get_state())
    assert b.time == a.time
    c1, p1, x1 = a.get_history()
    c2, p2, x2 = b.get_history()
    np.testing.assert_array_equal(c1, c2)
    live = (np.arange(p1.size) % 24) < np.repeat(c1, 24)
    np.testing.assert_array_equal(p1[live], p2[live])
    np.testing.assert_array_equal(x1.reshape(-1, 3)[live], x2.reshape(-1, 3)[live])
    # the state file alone is the reference's format
    a.write_state_file(str(tmp_path / "s.bin"))
    np.testing.assert_array_equal(read_state_file(str(tmp_path / "s.bin")).reshape(-1), a.get_state())
    frame = a.pack_frame([1.0, 2.0, 3.0, 4.0, 5.0])
    np.testing.assert_array_equal(frame[:3 * a.n], a.get_positions())
    # a state file that is not the one the sidecar was written with is refused, even
    # with the same grain count (a crash between the two renames leaves that pair)
    a.write_state_file(path)
    with pytest.raises(WorldError, match="another state file"):
        ParticleDynamics.from_checkpoint(cfg, path)
    assert frame[3 * a.n] == np.float32(a.time)
    np.testing.assert_array_equal(frame[3 * a.n + 1:], [1, 2, 3, 4, 5])
    a.close(); b.close()


def test_async_io_loop_matches_the_synchronous_one():
    from test_gpu_parity import packed_poly
    cfg, st, rad = packed_poly(n=1200, seed=41, mu=0.5)
    a = ParticleDynamics(cfg, state=st, radius=rad)
    b = ParticleDynamics(cfg, state=st, radius=rad)
    a.advance(5)
    b.advance(5)
    host = a.get_state()
    rng = np.random.default_rng(2)
    states = [host + rng.normal(0, 1e-6, host.shape).astype(np.float32) for _ in range(4)]
    outs_sync, outs_async = [], [np.empty(3 * a.n, np.float32) for _ in range(4)]
    for s_ in states:
        a.set_state(s_)
        a.advance(1)
        outs_sync.append(a.get_positions())
    check(lib.wd_io_join(b.handle))
    for k, s_ in enumerate(states):
        check(lib.wd_set_state_async(b.handle, ptr(s_)))
        check(lib.wd_step(b.handle, 1))
        check(lib.wd_get_positions_async(b.handle, ptr(outs_async[k])))
    check(lib.wd_synchronize(b.handle))
    for x, y in zip(outs_sync, outs_async):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    a.close(); b.close()


def test_grain_energies_sum_to_the_total_over_any_partition():
    from test_gpu_parity import packed_poly
    cfg, st, rad = packed_poly(n=2000, seed=8, mu=0.5)
    sim = ParticleDynamics(cfg, state=st, radius=rad)
    sim.advance(30)
    e = sim.grain_energies()
    total = sim.compute_total_energy()
    assert e.shape == (sim.n,)
    assert float(np.sum(e)) == pytest.approx(total, rel=1e-12)
    rng = np.random.default_rng(0)
    part = rng.integers(0, 3, sim.n)
    assert sum(float(np.sum(e[part == k])) for k in range(3)) == pytest.approx(total, rel=1e-12)
    sim.close()
