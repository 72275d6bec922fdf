"""world_b200: the world DEM step for NVIDIA B200 (sm_100a).

The compute path is libworld_b200.so (CUDA kernels + C ABI, include/world_b200.h);
this package is its Python face: SimConfig / load_config with the reference's YAML
schema, ParticleDynamics with the reference's step interface, SceneBatch (many
scenes in one step), seeded scene generators, and state / dataset file formats.

The library is loaded on first use of a name that needs it (PEP 562 module
__getattr__), so the pure-numpy modules (world_b200.scenes, world_b200.dataset_io)
import without it; every compute entry point still fails loudly when it is missing.
"""
from __future__ import annotations

import importlib

_LAZY = {
    "ParticleDynamics": ("particle_dynamics", "ParticleDynamics"),
    "SceneBatch": ("batch", "SceneBatch"),
    "SceneRange": ("batch", "SceneRange"),
    "SimConfig": ("config", "SimConfig"),
    "load_config": ("config", "load_config"),
    "WorldError": ("_lib", "WorldError"),
    "WD_HIST_CAP": ("_lib", "WD_HIST_CAP"),
    "lib": ("_lib", "lib"),
}

__all__ = sorted(_LAZY)


def __getattr__(name: str):
    try:
        module, attr = _LAZY[name]
    except KeyError:
        raise AttributeError(f"module 'world_b200' has no attribute '{name}'") from None
    value = getattr(importlib.import_module(f".{module}", __name__), attr)
    globals()[name] = value
    return value


def __dir__():
    return sorted(set(globals()) | set(_LAZY))
