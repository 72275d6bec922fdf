"""The reference's own CUDA step (src/*.cu compiled for sm_100a, oracle/_ref) against
libworld_b200 on the same GPU, the same input bytes and the same config.

Workload: the 2^20-grain column collapse in compat mode, the only physics the
reference runs: one radius (d = 5 mm), material-table mass, viscous friction
(mu = 0.5), max_force = k_n r = 250 N, restitution 0.5, dt = 1e-5 s, semi-implicit
Euler, 453 x 453 x 226 cells (7.0 mm), 8 grains per cell. The reference's take_step()
is synchronous (a device sync after every kernel, src/kernel.cu:31-38), so it is timed
by the host clock; ours by CUDA events around graph launches. Neither flushes L2.

Printed with `-s`: both rates and their ratio. The bar: ours faster, per-step search
and Verlet lists alike, and the same trajectory to FP32 round-off (the reference sums
forces in atomic slot order, ours in a fixed order).
"""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import scaled_error
from scale_cases import compat_column
from world_b200 import ParticleDynamics, load_config

pytestmark = pytest.mark.gpu


def _compat_collapse(tmp_path):
    yaml_path, _ = compat_column(tmp_path, 1 << 20, cic=128, cell=7.0e-3)
    return yaml_path


def _ours(yaml_path, skin, warm, steps, tune):
    import torch
    cfg = load_config(str(yaml_path))
    cfg.neighbor_skin = skin
    sim = ParticleDynamics(cfg)
    if tune:
        sim.autotune(steps=20)
    sim.advance(warm)
    sim.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.advance(steps)
    e1.record(stream)
    e1.synchronize()
    rate = sim.n * steps / (e0.elapsed_time(e1) / 1e3)
    state = sim.get_state()
    sim.close()
    return rate, state


def test_faster_than_the_reference_step_on_this_gpu(tmp_path):
    from oracle.oracle import ReferenceSim
    if not ReferenceSim.available():
        pytest.fail("oracle/_ref/libref_world.so missing (oracle/build.py builds it)")
    yaml_path = _compat_collapse(tmp_path)
    warm, steps = 20, 300

    ref = ReferenceSim(str(yaml_path))
    n = ref.n
    ref.step(warm)
    t0 = time.perf_counter()
    ref.step(steps)
    ref_rate = n * steps / (time.perf_counter() - t0)
    ref_state = ref.state()
    ref.close()

    searched, st_s = _ours(yaml_path, 0.0, warm, steps, tune=False)
    tuned, st_t = _ours(yaml_path, 0.0, warm, steps, tune=True)
    print(f"\nreference step (sm_100a build of src/*.cu): {ref_rate:.3e} grain-steps/s")
    print(f"libworld_b200, grid search every step:      {searched:.3e} grain-steps/s "
          f"({searched / ref_rate:.1f}x)")
    print(f"libworld_b200, autotuned (Verlet lists):    {tuned:.3e} grain-steps/s "
          f"({tuned / ref_rate:.1f}x)")
    assert n == 1 << 20
    assert searched > ref_rate and tuned > ref_rate
    # the schedule does not change the arithmetic
    np.testing.assert_array_equal(st_s, st_t)
    # same trajectory as the reference to FP32 round-off after 320 steps
    s, r = st_s.reshape(-1, 6), ref_state.reshape(-1, 6)
    assert scaled_error(s[:, :3], r[:, :3]) <= 1e-5
    assert scaled_error(s[:, 3:], r[:, 3:]) <= 1e-4
