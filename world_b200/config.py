"""SimConfig and load_config, backed by the library's own loader.

Mirrors the reference's SimConfig struct (src/sim_config.h:64-200): the same member
names (`cfg.collision_grid_size_x`, `cfg.physics.friction`, `cfg.domain.x_min`,
`cfg.masses`, ...) with the same defaults, and load_config(path)
(src/sim_config.cpp:153-195) with the same YAML-subset semantics. Values live in the
C library's wd_config, so Python, C++ and the YAML files all go through one parser.
"""
from __future__ import annotations

import ctypes
from typing import Any

from . import _lib
from ._lib import check, lib

# member -> (section, key, type); nested members are "physics.x" / "domain.x"
FIELDS: dict[str, tuple[str, str, type]] = {
    "dt": ("simulation", "dt", float),
    "collision_grid_size_x": ("simulation", "collision_grid_size_x", int),
    "collision_grid_size_y": ("simulation", "collision_grid_size_y", int),
    "collision_grid_size_z": ("simulation", "collision_grid_size_z", int),
    "particles_per_cell": ("simulation", "particles_per_cell", int),
    "threads_per_block": ("simulation", "threads_per_block", int),
    "density_grid_size_x": ("simulation", "density_grid_size_x", int),
    "density_grid_size_y": ("simulation", "density_grid_size_y", int),
    "density_grid_size_z": ("simulation", "density_grid_size_z", int),
    "history": ("simulation", "history", bool),
    "neighbor_skin": ("simulation", "neighbor_skin", float),
    "domain.x_min": ("domain", "x_min", float),
    "domain.x_max": ("domain", "x_max", float),
    "domain.y_min": ("domain", "y_min", float),
    "domain.y_max": ("domain", "y_max", float),
    "domain.z_min": ("domain", "z_min", float),
    "domain.z_max": ("domain", "z_max", float),
    "physics.gravity": ("physics", "gravity", float),
    "physics.particle_radius": ("physics", "particle_radius", float),
    "physics.max_force": ("physics", "max_force", float),
    "physics.floor_z": ("physics", "floor_z", float),
    "physics.ceiling_z": ("physics", "ceiling_z", float),
    "physics.wall_x_min": ("physics", "wall_x_min", float),
    "physics.wall_x_max": ("physics", "wall_x_max", float),
    "physics.wall_y_min": ("physics", "wall_y_min", float),
    "physics.wall_y_max": ("physics", "wall_y_max", float),
    "physics.restitution": ("physics", "restitution", float),
    "physics.friction": ("physics", "friction", float),
    "physics.normal_stiffness": ("physics", "normal_stiffness", float),
    "physics.tangential_stiffness": ("physics", "tangential_stiffness", float),
    "physics.density": ("physics", "density", float),
    "masses": ("materials", "masses", list),
    "init_type": ("initialization", "type", str),
    "init_state_path": ("initialization", "state_path", str),
    "init_x0": ("initialization", "x0", float),
    "init_y0": ("initialization", "y0", float),
    "init_z0": ("initialization", "z0", float),
    "init_vx0": ("initialization", "vx0", float),
    "init_vy0": ("initialization", "vy0", float),
    "init_vz0": ("initialization", "vz0", float),
    "init_jitter": ("initialization", "jitter", float),
    "init_seed": ("initialization", "seed", int),
    "init_perturbation": ("initialization", "perturbation", float),
    "init_perturbation_seed": ("initialization", "perturbation_seed", int),
    "cube_length_x": ("initialization", "cube_length_x", float),
    "cube_length_y": ("initialization", "cube_length_y", float),
    "cube_length_z": ("initialization", "cube_length_z", float),
    "two_particle_separation": ("initialization", "two_particle_separation", float),
    "particle_material": ("initialization", "particle_material", int),
    "num_triangles": ("rendering", "num_triangles", int),
    "port": ("drivers", "port", int),
    "steps_per_frame": ("drivers", "steps_per_frame", int),
    "profiling_outer_iters": ("drivers", "profiling_outer_iters", int),
    "profiling_steps_per_iter": ("drivers", "profiling_steps_per_iter", int),
    "kernel_timing": ("drivers", "kernel_timing", bool),
    "sweep_dt": ("sweep", "dt", list),
    "sweep_max_force": ("sweep", "max_force", list),
    "sweep_restitution": ("sweep", "restitution", list),
    "stability_mode": ("stability", "mode", str),
    "stability_sim_time": ("stability", "sim_time", float),
    "stability_acceleration_cutoff": ("stability", "acceleration_cutoff", float),
    "stability_steps_per_steadiness_check": ("stability", "steps_per_steadiness_check", int),
    "model_problem_sim_time": ("model_problem", "sim_time", float),
    "dataset_sim_time": ("dataset", "sim_time", float),
    "dataset_checkpoints": ("dataset", "checkpoints", int),
    "time_integrator": ("time_integration", "solver", str),
    "picard_iterations": ("time_integration", "picard_iterations", int),
    "picard_tolerance": ("time_integration", "picard_tolerance", float),
}


def _to_text(value: Any, typ: type) -> str:
    if typ is bool:
        return "true" if value else "false"
    if typ is list:
        return "[" + ", ".join(repr(float(v)) for v in value) + "]"
    if typ is float:
        return repr(float(value))
    return str(value)


def _from_text(text: str, typ: type) -> Any:
    if typ is bool:
        return text == "true"
    if typ is int:
        return int(text)
    if typ is float:
        return float(text)
    if typ is list:
        inner = text.strip()[1:-1].strip()
        return [float(v) for v in inner.split(",")] if inner else []
    return text


class _Section:
    def __init__(self, cfg: "SimConfig", prefix: str):
        object.__setattr__(self, "_cfg", cfg)
        object.__setattr__(self, "_prefix", prefix)

    def __getattr__(self, name: str) -> Any:
        return self._cfg._get_field(f"{self._prefix}.{name}")

    def __setattr__(self, name: str, value: Any) -> None:
        self._cfg._set_field(f"{self._prefix}.{name}", value)


class SimConfig:
    """The reference's SimConfig, with its defaults (src/sim_config.h:68-199)."""

    def __init__(self, _handle: int | None = None):
        h = ctypes.c_void_p()
        if _handle is None:
            check(lib.wd_config_create(ctypes.byref(h)))
        else:
            h = ctypes.c_void_p(_handle)
        object.__setattr__(self, "_h", h)

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.wd_config_destroy(h)
            object.__setattr__(self, "_h", None)

    def copy(self) -> "SimConfig":
        out = ctypes.c_void_p()
        check(lib.wd_config_copy(self._h, ctypes.byref(out)))
        return SimConfig(_handle=out.value)

    # raw section.key access (YAML text semantics)
    def set(self, section: str, key: str, value: Any) -> int:
        text = value if isinstance(value, str) else _to_text(value, type(value) if not isinstance(value, (list, tuple)) else list)
        return check(lib.wd_config_set(self._h, section.encode(), key.encode(), text.encode()))

    def get(self, section: str, key: str) -> str:
        buf = ctypes.create_string_buffer(4096)
        check(lib.wd_config_get(self._h, section.encode(), key.encode(), buf, len(buf)))
        return buf.value.decode()

    def load_yaml(self, path: str) -> int:
        return check(lib.wd_config_load_yaml(self._h, str(path).encode()))

    # reference member names
    def _get_field(self, name: str) -> Any:
        section, key, typ = FIELDS[name]
        return _from_text(self.get(section, key), typ)

    def _set_field(self, name: str, value: Any) -> None:
        section, key, typ = FIELDS[name]
        check(lib.wd_config_set(self._h, section.encode(), key.encode(),
                                _to_text(value, typ).encode()))

    @property
    def physics(self) -> _Section:
        return _Section(self, "physics")

    @property
    def domain(self) -> _Section:
        return _Section(self, "domain")

    def __getattr__(self, name: str) -> Any:
        if name in FIELDS:
            return self._get_field(name)
        raise AttributeError(name)

    def __setattr__(self, name: str, value: Any) -> None:
        if name in FIELDS:
            self._set_field(name, value)
        else:
            raise AttributeError(f"SimConfig has no member '{name}'")

    def as_dict(self) -> dict[str, Any]:
        return {name: self._get_field(name) for name in FIELDS}


def load_config(path: str) -> SimConfig:
    """Defaults, overridden by the keys present in the YAML file at `path`."""
    cfg = SimConfig()
    cfg.load_yaml(path)
    return cfg


__all__ = ["SimConfig", "load_config", "FIELDS"]
_ = _lib
