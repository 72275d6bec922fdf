"""world_b200: the world DEM step for NVIDIA B200 (sm_100a).

The compute path is libworld_b200.so (CUDA kernels + C ABI, include/world_b200.h);
this package is its Python face: SimConfig / load_config with the reference's YAML
schema, ParticleDynamics with the reference's step interface, SceneBatch (many
scenes in one step), seeded scene generators, and state / dataset file formats.
"""
from ._lib import WD_HIST_CAP, WorldError, lib
from .config import SimConfig, load_config
from .particle_dynamics import ParticleDynamics
from .batch import SceneBatch, SceneRange

__all__ = ["ParticleDynamics", "SceneBatch", "SceneRange", "SimConfig", "load_config",
           "WorldError", "WD_HIST_CAP", "lib"]
