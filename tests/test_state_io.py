"""Initial states and the state file format (reference src/particle_dynamics.cu:128-235).

Host-only: the initial grains come from the library's host code (wd_initial_state).
"""
from __future__ import annotations

import numpy as np
import pytest

from world_b200 import SimConfig, WorldError
from world_b200.state_io import grain_properties, initial_state, read_state_file, write_state_file


def test_default_cube_lattice():
    cfg = SimConfig()
    st, mat = initial_state(cfg)
    # 0.2 / (2 * 0.01) = 10 per side -> 1000 grains (src/sim_config.h:98-101)
    assert st.shape == (1000, 6)
    assert (mat == 1).all()
    r = np.float32(0.01)
    # particle p = (i*10 + j)*10 + k at origin + lattice * 2 * 1.01 * r
    for p, (i, j, k) in [(0, (0, 0, 0)), (1, (0, 0, 1)), (10, (0, 1, 0)), (999, (9, 9, 9))]:
        want = [np.float32(o) + np.float32(l) * np.float32(2.0) * np.float32(1.01) * r
                for o, l in zip((-0.5, 0.0, 0.0), (i, j, k))]
        assert np.array_equal(st[p, :3], np.array(want, np.float32))
    assert (st[:, 3:] == 0).all()


def test_cube_jitter_is_seeded_and_perturbation_is_independent():
    a = SimConfig(); a.init_jitter = 0.3
    b = SimConfig(); b.init_jitter = 0.3
    c = SimConfig(); c.init_jitter = 0.3; c.init_seed = 7
    sa, _ = initial_state(a)
    sb, _ = initial_state(b)
    sc, _ = initial_state(c)
    assert np.array_equal(sa, sb)
    assert not np.array_equal(sa, sc)
    base = SimConfig()
    s0, _ = initial_state(base)
    dev = np.abs(sa[:, :3] - s0[:, :3])
    assert dev.max() <= 0.3 * 0.01 * 1.0001
    # perturbation: an independent stream on top of the jittered lattice
    d = SimConfig(); d.init_jitter = 0.3; d.init_perturbation = 0.01; d.init_perturbation_seed = 3
    sd, _ = initial_state(d)
    assert 0 < np.abs(sd[:, :3] - sa[:, :3]).max() <= 0.01 * 0.01 * 1.001


def test_cube_initial_velocity_on_every_grain():
    cfg = SimConfig()
    cfg.init_vx0, cfg.init_vy0, cfg.init_vz0 = 1.5, -0.5, 0.25
    st, _ = initial_state(cfg)
    assert np.array_equal(st[:, 3:], np.tile(np.float32([1.5, -0.5, 0.25]), (st.shape[0], 1)))


def test_two_and_single_particle():
    cfg = SimConfig(); cfg.init_type = "two_particles"
    st, mat = initial_state(cfg)
    assert st.shape == (2, 6)
    assert st[1, 2] == np.float32(np.float32(0.0) + np.float32(0.1))
    cfg = SimConfig(); cfg.init_type = "single_particle"; cfg.init_vz0 = 2.0
    st, _ = initial_state(cfg)
    assert st.shape == (1, 6) and st[0, 5] == np.float32(2.0)


def test_state_file_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    st = rng.normal(size=(37, 6)).astype(np.float32)
    path = tmp_path / "s.bin"
    write_state_file(path, st)
    raw = path.read_bytes()
    assert len(raw) == 4 + 37 * 24 and np.frombuffer(raw[:4], "<i4")[0] == 37
    assert np.array_equal(read_state_file(path), st)
    cfg = SimConfig(); cfg.init_type = "file"; cfg.init_state_path = str(path)
    got, mat = initial_state(cfg)
    assert np.array_equal(got, st) and (mat == cfg.particle_material).all()


@pytest.mark.parametrize("content,what", [(None, "could not open"), (b"\x00\x00\x00\x00", "bad particle count"),
                                          (np.int32(5).tobytes() + b"\x00" * 20, "short of")])
def test_state_file_errors_are_statuses(tmp_path, content, what):
    path = tmp_path / "s.bin"
    if content is not None:
        path.write_bytes(content)
    cfg = SimConfig(); cfg.init_type = "file"; cfg.init_state_path = str(path)
    with pytest.raises(WorldError) as e:
        initial_state(cfg)
    assert what in str(e.value) and e.value.status == -3


def test_grain_properties_table_and_density():
    cfg = SimConfig()
    mat = np.array([1, 1, 0], np.int32)
    r, m = grain_properties(cfg, mat)
    assert np.allclose(r, 0.01) and np.allclose(m, [0.04, 0.04, 0.0])
    cfg.physics.density = 2500.0
    r, m = grain_properties(cfg, mat, np.float32([0.0025, 0.003, 0.0025]))
    assert np.allclose(m, 2500 * 4 / 3 * np.pi * np.float64(r) ** 3, rtol=1e-6)


def test_checkpoint_reader_and_missing_sidecar(tmp_path):
    import ctypes
    from world_b200 import SimConfig, WorldError
    from world_b200._lib import check, lib
    from world_b200.state_io import read_checkpoint, write_state_file
    n = 5
    rng = np.random.default_rng(1)
    st = rng.random((n, 6)).astype(np.float32)
    path = tmp_path / "c.bin"
    write_state_file(path, st)
    h = ctypes.c_void_p()
    cfg = SimConfig()
    # a state file without its sidecar is not a checkpoint (checked before any device call)
    with pytest.raises(WorldError, match="sidecar"):
        check(lib.wd_create_from_checkpoint(cfg.handle, str(path).encode(), ctypes.byref(h)))
    with pytest.raises(WorldError, match="cannot read"):
        check(lib.wd_create_from_checkpoint(cfg.handle, str(tmp_path / "none.bin").encode(),
                                            ctypes.byref(h)))
    r, m = rng.random(n).astype(np.float32), rng.random(n).astype(np.float32)
    mat = np.arange(n, dtype=np.int32)
    cnt = np.array([0, 2, 1, 0, 3], np.int32)
    part = rng.integers(-6, n, n * 24).astype(np.int32)
    xi = rng.random(n * 24 * 3).astype(np.float32)
    with open(str(path) + ".sidecar", "wb") as f:
        f.write(b"WDCKPT01")
        f.write(np.array([1, 1], "<u4").tobytes())
        f.write(np.array([n], "<i8").tobytes())
        f.write(np.array([0.25, 1e-5], "<f4").tobytes())
        for a in (r, m, mat, cnt, part, xi):
            f.write(a.tobytes())
    ck = read_checkpoint(path)
    np.testing.assert_array_equal(ck["state"], st)
    assert ck["time"] == np.float32(0.25) and ck["dt"] == np.float32(1e-5)
    for k, a in (("radius", r), ("mass", m), ("material", mat), ("count", cnt),
                 ("partner", part), ("xi", xi)):
        np.testing.assert_array_equal(ck[k], a)
    with open(str(path) + ".sidecar", "ab") as f:
        f.write(b"\0")
    with pytest.raises(ValueError, match="trailing"):
        read_checkpoint(path)
