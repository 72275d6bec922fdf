"""The multi-rank host path of the batched workloads on CPU: world_size 2 over gloo.
Each rank takes its shard of the scenes (no exchange) and the per-scene results
come back to every rank through one all-reduce."""
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
