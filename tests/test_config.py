"""Config schema and YAML-subset semantics (reference src/sim_config.h, src/sim_config.cpp).

Host-only: no device is touched.
"""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

from world_b200 import SimConfig, WorldError, load_config
from world_b200._lib import WD_WARN_DEFAULTS, WD_WARN_UNKNOWN_KEY

# Built-in defaults of the reference's SimConfig (src/sim_config.h:68-199).
REFERENCE_DEFAULTS = {
    "dt": 0.0001, "collision_grid_size_x": 32, "collision_grid_size_y": 32,
    "collision_grid_size_z": 32, "particles_per_cell": 64, "threads_per_block": 256,
    "density_grid_size_x": 32, "density_grid_size_y": 32, "density_grid_size_z": 32,
    "domain.x_min": -1.0, "domain.x_max": 1.0, "domain.y_min": -1.0, "domain.y_max": 1.0,
    "domain.z_min": -1.0, "domain.z_max": 1.0,
    "physics.gravity": 9.81, "physics.particle_radius": 0.01, "physics.max_force": 100.0,
    "physics.floor_z": -1.0, "physics.ceiling_z": 1.0, "physics.wall_x_min": -1.0,
    "physics.wall_x_max": 1.0, "physics.wall_y_min": -1.0, "physics.wall_y_max": 1.0,
    "physics.restitution": 0.3, "physics.friction": 0.5,
    "masses": [0.0, 0.04], "init_type": "cube", "init_state_path": "",
    "init_x0": -0.5, "init_y0": 0.0, "init_z0": 0.0, "init_vx0": 0.0, "init_vy0": 0.0,
    "init_vz0": 0.0, "init_jitter": 0.0, "init_seed": 12345, "init_perturbation": 0.0,
    "init_perturbation_seed": 1, "cube_length_x": 0.2, "cube_length_y": 0.2,
    "cube_length_z": 0.2, "two_particle_separation": 0.1, "particle_material": 1,
    "num_triangles": 20, "port": 8081, "steps_per_frame": 10, "profiling_outer_iters": 10,
    "profiling_steps_per_iter": 10, "kernel_timing": True, "sweep_dt": [],
    "sweep_max_force": [], "sweep_restitution": [], "stability_mode": "fixed_time",
    "stability_sim_time": 0.1, "stability_acceleration_cutoff": 0.01,
    "stability_steps_per_steadiness_check": 100, "model_problem_sim_time": 1.0,
    "dataset_sim_time": 2.0, "dataset_checkpoints": 10,
    "time_integrator": "semi_implicit_euler", "picard_iterations": 3,
}

# Keys this library adds; absent means the reference's behaviour.
EXTENSION_DEFAULTS = {"history": False, "physics.normal_stiffness": 0.0,
                      "physics.tangential_stiffness": 0.0, "physics.density": 0.0,
                      "picard_tolerance": 0.0}


def _get(cfg, name):
    if "." in name:
        sec, key = name.split(".")
        return getattr(getattr(cfg, sec), key)
    return getattr(cfg, name)


def test_defaults_match_reference():
    cfg = SimConfig()
    for name, want in {**REFERENCE_DEFAULTS, **EXTENSION_DEFAULTS}.items():
        got = _get(cfg, name)
        if isinstance(want, float):
            assert got == pytest.approx(np.float32(want), rel=1e-7), name
        elif isinstance(want, list):
            assert np.allclose(got, np.float32(want)), name
        else:
            assert got == want, name


def test_yaml_sections_lists_comments(tmp_path):
    p = tmp_path / "c.yaml"
    p.write_text(
        "# leading comment\n"
        "simulation:\n"
        "  dt: 0.001   # trailing comment\n"
        "  collision_grid_size_x: 100\n"
        "\n"
        "physics:\n"
        "  friction: 0.25\n"
        "materials:\n"
        "  masses: [0.0, 0.8, 1.5]\n"
        "initialization:\n"
        "  type: \"single_particle\"\n"
        "  state_path: 'dir/state.bin'\n"
        "drivers:\n"
        "  kernel_timing: false\n"
        "sweep:\n"
        "  dt: [1e-4, 2e-4]\n")
    cfg = load_config(str(p))
    assert cfg.dt == pytest.approx(np.float32(0.001))
    assert cfg.collision_grid_size_x == 100
    assert cfg.collision_grid_size_y == 32
    assert cfg.physics.friction == pytest.approx(0.25)
    assert np.allclose(cfg.masses, [0.0, 0.8, 1.5])
    assert cfg.init_type == "single_particle"
    assert cfg.init_state_path == "dir/state.bin"
    assert cfg.kernel_timing is False
    assert np.allclose(cfg.sweep_dt, [1e-4, 2e-4])


def test_missing_file_keeps_defaults(tmp_path):
    cfg = SimConfig()
    assert cfg.load_yaml(str(tmp_path / "absent.yaml")) == WD_WARN_DEFAULTS
    assert cfg.collision_grid_size_x == 32


def test_unknown_key_warns_and_rest_loads(tmp_path):
    p = tmp_path / "c.yaml"
    p.write_text("physics:\n  no_such_key: 3\n  gravity: 1.5\nnowhere:\n  x: 1\n")
    cfg = SimConfig()
    assert cfg.load_yaml(str(p)) == WD_WARN_UNKNOWN_KEY
    assert cfg.physics.gravity == pytest.approx(1.5)


def test_malformed_line_is_skipped(tmp_path):
    p = tmp_path / "c.yaml"
    p.write_text("simulation:\n  this line has no colon\n  dt: 0.5\n")
    cfg = load_config(str(p))
    assert cfg.dt == pytest.approx(0.5)


def test_unparsable_value_is_an_error_not_an_abort(tmp_path):
    p = tmp_path / "c.yaml"
    p.write_text("simulation:\n  dt: fast\n")
    with pytest.raises(WorldError) as e:
        load_config(str(p))
    assert "dt" in str(e.value)


def test_solver_name_is_kept_verbatim(tmp_path):
    # the reference stores time_integration.solver without unquoting
    # (src/sim_config.cpp:148): a quoted name is not "semi_implicit_euler"
    p = tmp_path / "c.yaml"
    p.write_text('time_integration:\n  solver: "semi_implicit_euler"\n  picard_iterations: 5\n')
    cfg = load_config(str(p))
    assert cfg.time_integrator == '"semi_implicit_euler"'
    assert cfg.picard_iterations == 5


def test_stoi_prefix_semantics():
    cfg = SimConfig()
    cfg.set("simulation", "particles_per_cell", "12abc")   # std::stoi reads the prefix
    assert cfg.particles_per_cell == 12


def test_extension_keys_round_trip(tmp_path):
    p = tmp_path / "c.yaml"
    p.write_text("simulation:\n  history: true\nphysics:\n  normal_stiffness: 1e5\n"
                 "  tangential_stiffness: 3e4\n  density: 2500\n"
                 "time_integration:\n  picard_tolerance: 1e-6\n")
    cfg = load_config(str(p))
    assert cfg.history is True
    assert cfg.physics.normal_stiffness == pytest.approx(1e5)
    assert cfg.physics.tangential_stiffness == pytest.approx(3e4)
    assert cfg.physics.density == pytest.approx(2500.0)
    assert cfg.picard_tolerance == pytest.approx(1e-6)


def test_copy_is_independent():
    a = SimConfig()
    b = a.copy()
    b.physics.friction = 0.1
    assert a.physics.friction == pytest.approx(0.5)


def _reference_root() -> str:
    """The reference tree the oracle's build recipe reads (oracle/build.py)."""
    from oracle import build as oracle_build
    return os.path.dirname(oracle_build.REFERENCE_SRC.rstrip("/"))


@pytest.mark.skipif(not os.path.isdir(_reference_root()), reason="reference tree not present")
def test_every_reference_yaml_loads_without_unknown_keys():
    files = [f for f in glob.glob(os.path.join(_reference_root(), "**", "*.yaml"), recursive=True)]
    assert files
    for f in files:
        cfg = SimConfig()
        assert cfg.load_yaml(f) == 0, f
