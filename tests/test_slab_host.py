"""The slab decomposition (world_b200/slab.py) on CPU: two gloo ranks, the oracle as
each rank's local step, against the oracle stepping the whole scene in one process.
The owned grains' states and springs must be the single-process ones bit for bit after
every check, grains must migrate across the cut, and momentum is an FP64 all-reduce."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from world_b200.slab import cell_x, slab_cuts


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, steps, out_dir):
    import datetime
    import sys
    sys.path[:0] = [os.path.dirname(os.path.abspath(__file__))]
    import torch.distributed as dist
    from slab_cases import OracleStepper, sheared_pack
    from world_b200.scenes import grain_properties
    from world_b200.slab import SlabDomain
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        cfg, st, rad = sheared_pack()
        _, mass = grain_properties(cfg, np.full(st.shape[0], cfg.particle_material, np.int32), rad)
        dom = SlabDomain(cfg, st, rad, mass, OracleStepper(cfg))
        for k in range(steps // 20):
            dom.step(20)
            state, (cnt, part, xi) = dom.gather()
            if rank == 0:
                np.savez(os.path.join(out_dir, f"chk{k}.npz"), state=state, cnt=cnt,
                         part=part, xi=xi, momentum=dom.momentum())
            else:
                dom.momentum()
        moved = np.array([dom.migrated], np.int64)
        np.save(os.path.join(out_dir, f"migrated{rank}.npy"), moved)
        np.save(os.path.join(out_dir, f"owned{rank}.npy"), np.array([dom.owned.k]))
    finally:
        dist.destroy_process_group()


def test_two_slabs_equal_the_single_process_step(tmp_path, oracle_for):
    from slab_cases import sheared_pack
    steps, world = 80, 2
    mp.start_processes(_rank_main, args=(world, _free_port(), steps, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    cfg, st, rad = sheared_pack()
    orc = oracle_for(cfg, st, radius=rad)
    for k in range(steps // 20):
        orc.step(20)
        z = np.load(tmp_path / f"chk{k}.npz")
        np.testing.assert_array_equal(z["state"].reshape(-1), orc.state)
        np.testing.assert_array_equal(z["cnt"], orc.hcnt)
        live = (np.arange(24)[None, :] < orc.hcnt[:, None]).reshape(-1)
        np.testing.assert_array_equal(z["part"].reshape(-1)[live], orc.hpart[live])
        np.testing.assert_array_equal(z["xi"].reshape(-1, 3)[live], orc.hxi.reshape(-1, 3)[live])
        np.testing.assert_allclose(z["momentum"], orc.momentum(), rtol=1e-12, atol=1e-15)
    assert orc.hcnt.sum() > 500                        # springs were carried
    migrated = sum(int(np.load(tmp_path / f"migrated{r}.npy")[0]) for r in range(world))
    assert migrated > 20                               # grains changed slab
    owned = [int(np.load(tmp_path / f"owned{r}.npy")[0]) for r in range(world)]
    assert sum(owned) == st.shape[0] and min(owned) > 0


def test_cuts_balance_and_cover_the_grid():
    rng = np.random.default_rng(0)
    x = rng.normal(0.0, 0.1, 100000).astype(np.float32)
    cols = cell_x(x, -1.0, 1.0, 200)
    for ranks in (1, 2, 3, 8):
        c = slab_cuts(cols, 200, ranks)
        assert c[0] == 0 and c[-1] == 200 and np.all(np.diff(c) >= 1)
        load = np.array([((cols >= c[r]) & (cols < c[r + 1])).sum() for r in range(ranks)])
        assert load.sum() == x.size
        assert load.max() - load.min() <= np.bincount(cols).max() * 2
    with pytest.raises(ValueError):
        slab_cuts(cols, 200, 201)


def test_cell_x_is_the_reference_expression():
    x = np.array([-1.0, -0.99, 0.0, 0.3333333, 0.999, 1.0, 2.0, np.nan], np.float32)
    got = cell_x(x, -1.0, 1.0, 6)
    f32 = np.float32
    t = ((x - f32(-1)) / (f32(1) - f32(-1))) * f32(6)
    want = np.clip(np.nan_to_num(np.trunc(t), nan=0).astype(np.int64), 0, 5)
    np.testing.assert_array_equal(got, want)
