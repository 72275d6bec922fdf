"""The slab decomposition with libworld_b200 as each rank's local step: two processes
sharing one GPU, exchanging over gloo (their kernels never wait on each other: every
exchange is a host message between steps). Against the library stepping the whole scene
in one process: owned grains' states and springs bit for bit, the FP64 all-reduced
energy (per-grain terms, each pair carried by its smaller-id grain) and momentum.

Scenes: the sheared packing (grains cross the cut every few steps) and the 32,768-grain
column 12,000 steps in (collapsing onto the floor, contacts across the cut).
Multi-GPU runs are not available here: unmeasured on hardware beyond one GPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene(name, tmp):
    from slab_cases import sheared_pack
    from world_b200.scenes import column_collapse
    if name == "sheared":
        cfg, st, rad = sheared_pack()
        return cfg, st, rad, None, 80
    sc = column_collapse(32768, diameters="uniform", cic=64)
    z = np.load(os.path.join(tmp, "column.npz"))
    return sc.cfg, z["state"].reshape(-1, 6), sc.radius, (z["cnt"], z["part"], z["xi"]), 50


def _rank_main(rank, world, port, name, tmp):
    import datetime
    import sys
    sys.path[:0] = [os.path.dirname(os.path.abspath(__file__))]
    import torch.distributed as dist
    from world_b200.scenes import grain_properties
    from world_b200.slab import LibraryStepper, SlabDomain
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    stepper = None
    try:
        cfg, st, rad, springs, steps = _scene(name, tmp)
        cfg.kernel_timing = False
        _, mass = grain_properties(cfg, np.full(st.shape[0], cfg.particle_material, np.int32), rad)
        stepper = LibraryStepper(cfg)
        dom = SlabDomain(cfg, st, rad, mass, stepper, springs=springs)
        dom.step(steps)
        state, rows = dom.gather()
        energy, momentum = dom.total_energy(), dom.momentum()
        if rank == 0:
            np.savez(os.path.join(tmp, f"{name}_slab.npz"), state=state, cnt=rows[0],
                     part=rows[1], xi=rows[2], energy=energy, momentum=momentum)
        np.save(os.path.join(tmp, f"{name}_migrated{rank}.npy"), np.array([dom.migrated]))
    finally:
        if stepper is not None:
            stepper.close()
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["sheared", "column"])
def test_two_slabs_on_one_gpu_equal_the_single_process_step(tmp_path, name):
    from world_b200 import ParticleDynamics
    tmp = str(tmp_path)
    if name == "column":
        from world_b200.scenes import column_collapse
        sc = column_collapse(32768, diameters="uniform", cic=64)
        sc.cfg.kernel_timing = False
        pre = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
        pre.advance(12000)
        cnt, part, xi = pre.get_history()
        np.savez(os.path.join(tmp, "column.npz"), state=pre.get_state(), cnt=cnt, part=part, xi=xi)
        pre.close()
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), name, tmp), nprocs=world,
                       join=True, start_method="spawn")
    cfg, st, rad, springs, steps = _scene(name, tmp)
    cfg.kernel_timing = False
    one = ParticleDynamics(cfg, state=st, radius=rad)
    if springs is not None:
        one.set_history(*springs)
    one.advance(steps)
    z = np.load(os.path.join(tmp, f"{name}_slab.npz"))
    np.testing.assert_array_equal(z["state"].reshape(-1), one.get_state())
    cnt, part, xi = one.get_history()
    np.testing.assert_array_equal(z["cnt"], cnt)
    live = (np.arange(24)[None, :] < cnt[:, None]).reshape(-1)
    np.testing.assert_array_equal(z["part"].reshape(-1)[live], part[live])
    np.testing.assert_array_equal(z["xi"].reshape(-1, 3)[live], xi.reshape(-1, 3)[live])
    assert float(z["energy"]) == pytest.approx(one.compute_total_energy(), rel=1e-12)
    np.testing.assert_allclose(z["momentum"], one.compute_momentum(), rtol=1e-12, atol=1e-15)
    assert cnt.sum() > 500
    migrated = sum(int(np.load(os.path.join(tmp, f"{name}_migrated{r}.npy"))[0]) for r in range(world))
    if name == "sheared":
        assert migrated > 20
    one.close()
