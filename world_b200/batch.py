"""SceneBatch: many independent scenes stepped as one (wd_create_batch).

The reference runs an ensemble or a dataset design one ParticleDynamics at a time
(src/dataset.cpp:163-232 loops over design rows, src/chaos.cpp:176-206 over
perturbed members). Here the scenes share one handle: one neighbor search, one
contact launch and one integration per step for all of them. Scene k owns the grain
ids ``ranges[k].first ... first + count`` in every array the ParticleDynamics
interface returns, and the float range ``4 * node_first ... 4 * (node_first + nodes)``
of ``host_density_grid`` (channel-major, like a single scene's grid). Each scene's
trajectory, candidates, density field and energy equal its solo run bit for bit.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from ._lib import check, lib, ptr
from .config import SimConfig
from .particle_dynamics import ParticleDynamics


@dataclass(frozen=True)
class SceneRange:
    first: int        # first grain id of the scene
    count: int        # grains in the scene
    node_first: int   # first density node of the scene
    nodes: int        # density nodes of the scene


def shard_scenes(counts: Sequence[int], ranks: int) -> list[list[int]]:
    """Scenes shared out over ranks, balanced by grain count: largest scene first to
    the least-loaded rank (ties to the lower rank). Each rank's list is ascending.
    Every rank computes the same answer from the same counts, with no exchange."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    if len(counts) < ranks:
        raise ValueError(f"{len(counts)} scenes cannot be shared over {ranks} ranks")
    load = [0] * ranks
    out: list[list[int]] = [[] for _ in range(ranks)]
    for k in sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i)):
        r = min(range(ranks), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += int(counts[k])
    return [sorted(x) for x in out]


def _ptr_array(arrays: Sequence[Optional[np.ndarray]]):
    if all(a is None for a in arrays):
        return None, []
    keep = list(arrays)
    arr = (ctypes.c_void_p * len(keep))(*[None if a is None else a.ctypes.data for a in keep])
    return arr, keep


class SceneBatch(ParticleDynamics):
    """ParticleDynamics over several scenes. ``config`` is scene 0's configuration."""

    def __init__(self, configs: Sequence[SimConfig], states: Sequence[np.ndarray], *,
                 radii: Optional[Sequence[Optional[np.ndarray]]] = None,
                 masses: Optional[Sequence[Optional[np.ndarray]]] = None,
                 materials: Optional[Sequence[Optional[np.ndarray]]] = None):
        S = len(configs)
        if S < 1 or len(states) != S:
            raise ValueError("SceneBatch needs one state per config")
        self.configs = list(configs)
        self.config = self.configs[0]
        sts = [np.ascontiguousarray(s, dtype=np.float32).reshape(-1) for s in states]
        counts = np.array([s.size // 6 for s in sts], np.int64)

        def per_scene(seq, dtype, name):
            if seq is None:
                return [None] * S
            if len(seq) != S:
                raise ValueError(f"{name} needs one entry per scene")
            out = []
            for k, a in enumerate(seq):
                if a is None:
                    out.append(None)
                    continue
                a = np.ascontiguousarray(a, dtype=dtype).reshape(-1)
                if a.size != counts[k]:
                    raise ValueError(f"{name}[{k}] has {a.size} entries for {counts[k]} grains")
                out.append(a)
            return out

        rad = per_scene(radii, np.float32, "radii")
        ms = per_scene(masses, np.float32, "masses")
        mat = per_scene(materials, np.int32, "materials")
        cfg_arr = (ctypes.c_void_p * S)(*[c.handle for c in self.configs])
        st_arr = (ctypes.c_void_p * S)(*[s.ctypes.data for s in sts])
        rad_arr, _k1 = _ptr_array(rad)
        ms_arr, _k2 = _ptr_array(ms)
        mat_arr, _k3 = _ptr_array(mat)
        h = ctypes.c_void_p()
        check(lib.wd_create_batch(cfg_arr, S, ptr(counts), st_arr, mat_arr, rad_arr, ms_arr,
                                  ctypes.byref(h)))
        self._attach(h)
        self.ranges = [self._range(k) for k in range(S)]

    @classmethod
    def from_scenes(cls, scenes) -> "SceneBatch":
        """From scene-generator outputs (objects with cfg, state and radius)."""
        return cls([s.cfg for s in scenes], [s.state for s in scenes],
                   radii=[s.radius for s in scenes])

    def _range(self, k: int) -> SceneRange:
        v = [ctypes.c_int64() for _ in range(4)]
        check(lib.wd_scene_range(self._h, k, *[ctypes.byref(x) for x in v]))
        return SceneRange(*(int(x.value) for x in v))

    @property
    def scenes(self) -> int:
        s = ctypes.c_int32()
        check(lib.wd_scene_count(self._h, ctypes.byref(s)))
        return int(s.value)

    # -- per-scene views of the batch-wide arrays ------------------------------------
    def split(self, per_grain: np.ndarray, width: int) -> list[np.ndarray]:
        """Cut an array of ``width`` values per grain id into the scenes' pieces."""
        a = np.asarray(per_grain).reshape(-1, width)
        return [a[r.first:r.first + r.count].reshape(-1) for r in self.ranges]

    def scene_states(self) -> list[np.ndarray]:
        return self.split(self.get_state(), 6)

    def scene_density_grids(self) -> list[np.ndarray]:
        self.compute_density_grid()
        g = self.host_density_grid
        return [g[4 * r.node_first:4 * (r.node_first + r.nodes)].copy() for r in self.ranges]

    def scene_energies(self) -> np.ndarray:
        out = np.empty(len(self.ranges), np.float64)
        check(lib.wd_compute_scene_energies(self._h, ptr(out)))
        return out

    def scene_momenta(self) -> np.ndarray:
        out = np.empty(3 * len(self.ranges), np.float64)
        check(lib.wd_compute_scene_momenta(self._h, ptr(out)))
        return out.reshape(-1, 3)

    # -- per-scene diagnostics and ensemble measures ---------------------------------
    def overflow_counts(self) -> np.ndarray:
        out = np.empty(len(self.ranges), np.int64)
        check(lib.wd_scene_overflow_counts(self._h, ptr(out)))
        return out

    def stability(self) -> np.ndarray:
        out = np.empty(len(self.ranges), np.int32)
        check(lib.wd_scene_stability(self._h, ptr(out)))
        return out.astype(bool)

    def freeze(self, scene: int, frozen: bool = True) -> None:
        """Stop (or restart) one scene: the step leaves its grains where they are."""
        check(lib.wd_freeze_scene(self._h, int(scene), 1 if frozen else 0))

    def chaos_metrics(self, reference_scene: int = 0) -> np.ndarray:
        """(scenes, 3): grain RMS separation, mass-field relative difference and
        centre-of-mass displacement (node units) of every scene from the reference
        scene, as the reference's chaos driver measures its members."""
        out = np.empty(3 * len(self.ranges), np.float64)
        check(lib.wd_chaos_metrics(self._h, int(reference_scene), ptr(out)))
        return out.reshape(-1, 3)


def gather_scene_values(local: np.ndarray, mine: Sequence[int], total: int, group=None) -> np.ndarray:
    """Per-scene results of every rank on every rank: ``local`` holds one row per
    scene in ``mine`` (this rank's shard, in order); the answer holds one row per
    scene of the whole ensemble. One all-reduce of a (total, width) FP64 array in
    which each row has a single non-zero contributor, so the sums are exact. Needs
    an initialised torch.distributed process group (gloo on CPU, NCCL on GPUs)."""
    import torch
    import torch.distributed as dist

    loc = np.asarray(local, np.float64).reshape(len(mine), -1)
    full = np.zeros((total, loc.shape[1]), np.float64)
    full[list(mine)] = loc
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(full).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()
