"""The batched workloads' multi-rank path with real steps: two processes on one GPU
(gloo), each stepping its shard of a SceneBatch (world_b200.batch.shard_scenes) as one
batch; the per-scene energies gathered over the ranks (gather_scene_values) equal those
of the unsharded batch stepped in one process, bit for bit (each scene reduces the same
way alone or in any batch)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

STEPS = 300


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _members():
    from world_b200.scenes import ensemble_set_b
    members = ensemble_set_b(scenes=7, seed=5, n_min=2048, n_max=16384)
    for m in members:
        m.cfg.neighbor_skin = 0.15 * 5e-3
    return members


def _rank_main(rank, world, port, tmp):
    import datetime
    import torch.distributed as dist
    from world_b200 import SceneBatch
    from world_b200.batch import gather_scene_values, shard_scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    try:
        members = _members()
        mine = shard_scenes([m.n for m in members], world)[rank]
        batch = SceneBatch.from_scenes([members[k] for k in mine])
        batch.advance(STEPS)
        local = np.concatenate([batch.scene_energies()[:, None], batch.scene_momenta()], 1)
        full = gather_scene_values(local, mine, len(members))
        if rank == 0:
            np.save(os.path.join(tmp, "gathered.npy"), full)
        batch.close()
    finally:
        dist.destroy_process_group()


def test_sharded_batch_equals_the_unsharded_batch(tmp_path):
    from world_b200 import SceneBatch
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    members = _members()
    batch = SceneBatch.from_scenes(members)
    batch.advance(STEPS)
    want = np.concatenate([batch.scene_energies()[:, None], batch.scene_momenta()], 1)
    got = np.load(tmp_path / "gathered.npy")
    np.testing.assert_array_equal(got, want)
    batch.close()
