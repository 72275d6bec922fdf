"""The reference's own tests (test/particle_dynamics_test.cpp:16-285), run against the
library on the GPU through the ParticleDynamics interface, written the way the
reference writes them (host_state edits pushed with device_state.copy_from_host)."""
from __future__ import annotations

import numpy as np
import pytest

from world_b200 import ParticleDynamics, SimConfig

pytestmark = pytest.mark.gpu


def test_runs_stably_for_fixed_iterations():
    sim = ParticleDynamics()
    for _ in range(100):
        sim.take_step()
    assert sim.is_stable()


def test_free_fall_matches_kinematics():
    sim = ParticleDynamics()
    hs = sim.host_state.reshape(-1, 6)
    hs[:, 3:] = 0.0
    sim.device_state.copy_from_host(sim.host_state)
    z0 = sim.host_state[2]
    steps = 100
    for _ in range(steps):
        sim.take_step()
    sim.unpack_state()
    dt = np.float32(sim.dt)
    expected = np.float32(-9.81) * dt * dt * np.float32(steps) * np.float32(steps + 1) / np.float32(2)
    assert abs((sim.positions[2] - z0) - expected) <= 1e-6


def test_particle_does_not_penetrate_floor():
    sim = ParticleDynamics()
    sim.host_state[:6] = [0.5, 0.5, -0.5, 0.0, 0.0, 0.0]
    sim.device_state.copy_from_host(sim.host_state)
    for _ in range(20000):
        sim.take_step()
    sim.unpack_state()
    assert sim.positions[2] >= -1.0 + 0.01 - 1e-3
    assert sim.is_stable()


def test_repeated_runs_are_deterministic():
    def run():
        sim = ParticleDynamics()
        for _ in range(50):
            sim.take_step()
        sim.unpack_state()
        return sim.positions.copy()
    assert np.array_equal(run(), run())


def test_grid_overflow_is_counted_and_stays_in_bounds():
    cfg = SimConfig()
    cfg.collision_grid_size_x = cfg.collision_grid_size_y = cfg.collision_grid_size_z = 1
    cfg.particles_per_cell = 2
    sim = ParticleDynamics(cfg)
    assert sim.n > cfg.particles_per_cell
    assert sim.grid_overflow_count() == 0
    sim.take_step()
    assert sim.grid_overflow_count() > 0
    sim.unpack_state()
    assert np.isfinite(sim.positions).all()


def test_total_energy_never_increases():
    sim = ParticleDynamics()
    previous = sim.compute_total_energy()
    initial = previous
    assert initial > 0
    tol = 1e-3 * initial
    for _ in range(12):
        for _ in range(100):
            sim.take_step()
        current = sim.compute_total_energy()
        assert current <= previous + tol
        previous = current
    assert previous < initial


def test_density_grid_conserves_total_mass():
    cfg = SimConfig(); cfg.init_jitter = 0.3
    sim = ParticleDynamics(cfg)
    for _ in range(250):
        sim.take_step()
    sim.compute_density_grid()
    deposited = sim.host_density_grid[:sim.density_grid_nodes()].astype(np.float64).sum()
    sim.unpack_state()
    expected = sum(float(sim.host_mass[m]) for m in sim.host_material)
    assert expected > 0
    assert abs(deposited - expected) <= 1e-4 * expected


def _single(x, y, z, size=32, v=(0.0, 0.0, 0.0)):
    cfg = SimConfig()
    cfg.init_type = "single_particle"
    cfg.density_grid_size_x = cfg.density_grid_size_y = cfg.density_grid_size_z = size
    cfg.init_x0, cfg.init_y0, cfg.init_z0 = x, y, z
    cfg.init_vx0, cfg.init_vy0, cfg.init_vz0 = v
    return cfg


def test_density_grid_puts_grain_on_node_at_single_node():
    cfg = _single(-0.5, 0.0, 0.5, size=5)
    sim = ParticleDynamics(cfg)
    sim.compute_density_grid()
    expected = (1 * 5 + 2) * 5 + 3
    m = float(sim.host_mass[cfg.particle_material])
    for node in range(sim.density_grid_nodes()):
        want = m if node == expected else 0.0
        assert abs(sim.host_density_grid[node] - want) <= 1e-6 * m


def test_density_grid_splits_cell_center_eight_ways():
    cfg = _single(-0.75, -0.25, 0.25, size=5)
    sim = ParticleDynamics(cfg)
    sim.compute_density_grid()
    m = float(sim.host_mass[cfg.particle_material])
    vals = sim.host_density_grid[:sim.density_grid_nodes()]
    nz = vals[vals > 1e-9]
    assert nz.size == 8
    assert np.allclose(nz, m / 8, atol=1e-5 * m)
    assert abs(vals.sum() - m) <= 1e-5 * m


def test_density_grid_momentum_matches_mass_times_velocity():
    cfg = _single(-0.5, 0.0, 0.0, v=(2.0, -3.0, 0.5))
    sim = ParticleDynamics(cfg)
    sim.compute_density_grid()
    nodes = sim.density_grid_nodes()
    m = float(sim.host_mass[cfg.particle_material])
    for a, v in enumerate((2.0, -3.0, 0.5)):
        got = sim.host_density_grid[(a + 1) * nodes:(a + 2) * nodes].astype(np.float64).sum()
        assert abs(got - m * v) <= 1e-4 * abs(m * v) + 1e-9


def test_cube_grains_receive_initial_velocity():
    cfg = SimConfig()
    cfg.init_vx0, cfg.init_vy0, cfg.init_vz0 = 1.5, -0.5, 0.25
    cfg.physics.gravity = 0.0
    sim = ParticleDynamics(cfg)
    assert sim.n > 1
    expected = np.float32([1.5, -0.5, 0.25])
    assert np.array_equal(sim.host_state.reshape(-1, 6)[:, 3:], np.tile(expected, (sim.n, 1)))
    before = sim.positions.copy()
    for _ in range(50):
        sim.take_step()
    sim.unpack_state()
    elapsed = sim.dt * 50
    for a in range(3):
        moved = sim.positions[a] - before[a]
        assert abs(moved - expected[a] * elapsed) <= 1e-4 * abs(expected[a] * elapsed) + 1e-6
