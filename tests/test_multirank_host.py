"""The multi-rank host path of the batched workloads on CPU: world_size 2 over gloo.
Each rank takes its shard of the scenes (no exchange) and the per-scene results
come back to every rank through one all-reduce: first with stand-in values, then with
every rank stepping its own scenes (the oracle as the local step)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from world_b200.batch import gather_scene_values, shard_scenes


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, counts, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shards = shard_scenes(counts, world)
        mine = shards[rank]
        # stand-in per-scene results: (energy, momentum x, y, z) from the scene index
        local = np.array([[k * 1.5 + 0.25, -k, k * k, 1e-300 * k] for k in mine])
        full = gather_scene_values(local, mine, len(counts))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), full)
        np.save(os.path.join(out_dir, f"shard{rank}.npy"), np.array(mine))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_gather(tmp_path):
    counts = [4096, 131072, 9000, 70000, 4100, 25000, 100000]
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), counts, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    want = np.array([[k * 1.5 + 0.25, -k, k * k, 1e-300 * k] for k in range(len(counts))])
    for r in range(world):
        np.testing.assert_array_equal(np.load(tmp_path / f"rank{r}.npy"), want)
    s0, s1 = (set(np.load(tmp_path / f"shard{r}.npy").tolist()) for r in range(world))
    assert s0 | s1 == set(range(len(counts))) and not (s0 & s1)
    load = [sum(counts[k] for k in s) for s in (s0, s1)]
    assert max(load) - min(load) <= max(counts)


def _shard_scenes_list():
    """Seven small columns of uneven size and friction (the batched workloads' kind)."""
    from world_b200.scenes import column_collapse
    sizes = [600, 1500, 800, 1200, 500, 1000, 700]
    return [column_collapse(n, diameters="uniform", mu=0.1 * (k % 6), seed=40 + k, cic=16)
            for k, n in enumerate(sizes)]


def _oracle_scene(scene):
    from oracle.oracle import OracleSim, lib as oracle_lib, params_from_config
    from world_b200.scenes import grain_properties
    oracle_lib().dem_set_num_threads(1)
    material = np.full(scene.n, scene.spec.particle_material, np.int32)
    radius, mass = grain_properties(scene.spec, material, scene.radius)
    return OracleSim(params_from_config(scene.spec), scene.state, radius, mass)


def _scene_values(scene, steps):
    sim = _oracle_scene(scene)
    sim.step(steps)
    return np.concatenate([[sim.energy()], sim.momentum()])


def _stepping_rank(rank, world, port, steps, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        scenes = _shard_scenes_list()
        mine = shard_scenes([sc.n for sc in scenes], world)[rank]
        local = np.array([_scene_values(scenes[k], steps) for k in mine]).reshape(-1, 4)
        full = gather_scene_values(local, mine, len(scenes))
        np.save(os.path.join(out_dir, f"stepped{rank}.npy"), full)
    finally:
        dist.destroy_process_group()


def test_two_ranks_step_their_shards():
    """Each rank steps only its own shard of the scenes (the oracle as the local step,
    every scene independent as in a SceneBatch); after the one FP64 all-reduce every
    rank holds each scene's energy and momentum exactly as one process stepping every
    scene gets them."""
    import tempfile
    steps, world = 60, 2
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_stepping_rank, args=(world, _free_port(), steps, out),
                           nprocs=world, join=True, start_method="spawn")
        got = [np.load(os.path.join(out, f"stepped{r}.npy")) for r in range(world)]
    want = np.array([_scene_values(sc, steps) for sc in _shard_scenes_list()])
    assert np.abs(want[:, 0]).min() > 0
    for g in got:
        np.testing.assert_array_equal(g, want)


def test_shards_are_balanced_and_deterministic():
    rng = np.random.default_rng(3)
    counts = np.exp(rng.uniform(np.log(4096), np.log(131072), 256)).astype(int).tolist()
    for ranks in (1, 2, 3, 8):
        a = shard_scenes(counts, ranks)
        assert a == shard_scenes(counts, ranks)
        flat = sorted(k for s in a for k in s)
        assert flat == list(range(256))
        load = [sum(counts[k] for k in s) for s in a]
        assert max(load) - min(load) <= max(counts)
    with pytest.raises(ValueError):
        shard_scenes([1, 2], 3)
