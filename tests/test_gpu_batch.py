"""Batched scenes (wd_create_batch) against the same scenes run one at a time.

Every scene of a batch must reproduce its solo run bit for bit: state, tangential
history, candidate and contact lists, density field, energy and momentum. The solo
runs are themselves pinned to the oracle by test_gpu_parity.py, so this pins the
batch to the oracle too.
"""
from __future__ import annotations

import numpy as np
import pytest

from world_b200 import ParticleDynamics, SceneBatch, SimConfig
from world_b200.scenes import column_collapse, perturbed_members
from world_b200.state_io import initial_state

from test_gpu_parity import packed_poly

pytestmark = pytest.mark.gpu


def _solo(cfg, state, radius, steps):
    sim = ParticleDynamics(cfg, state=state, radius=radius)
    sim.advance(steps)
    return sim


def _check_scene(batch: SceneBatch, k: int, solo: ParticleDynamics):
    r = batch.ranges[k]
    assert r.count == solo.n
    st = batch.scene_states()[k]
    np.testing.assert_array_equal(st, solo.get_state())
    # candidate and contact lists, global ids shifted back to the scene's own
    off, cand, contact = batch.debug_candidates()
    s_off, s_cand, s_contact = solo.debug_candidates()
    lo, hi = off[r.first], off[r.first + r.count]
    np.testing.assert_array_equal(off[r.first:r.first + r.count + 1] - lo, s_off)
    np.testing.assert_array_equal(cand[lo:hi] - r.first, s_cand)
    np.testing.assert_array_equal(contact[lo:hi], s_contact)
    grids = batch.scene_density_grids()
    solo.compute_density_grid()
    np.testing.assert_array_equal(grids[k], solo.host_density_grid)
    assert batch.scene_energies()[k] == solo.compute_total_energy()
    np.testing.assert_array_equal(batch.scene_momenta()[k], solo.compute_momentum())


def _check_history(batch: SceneBatch, k: int, solo: ParticleDynamics):
    r = batch.ranges[k]
    cnt, part, xi = batch.get_history()
    s_cnt, s_part, s_xi = solo.get_history()
    cap = s_part.size // solo.n
    np.testing.assert_array_equal(cnt[r.first:r.first + r.count], s_cnt)
    p = part[r.first * cap:(r.first + r.count) * cap].copy()
    live = (np.arange(p.size) % cap) < np.repeat(s_cnt, cap)
    grain = live & (p >= 0)
    p[grain] -= r.first
    np.testing.assert_array_equal(p[live], s_part[live])
    x = xi[3 * r.first * cap:3 * (r.first + r.count) * cap].reshape(-1, 3)
    np.testing.assert_array_equal(x[live], s_xi.reshape(-1, 3)[live])


def test_batch_history_scenes_match_solo():
    a = packed_poly(n=3000, seed=3, mu=0.5)
    b = packed_poly(n=1500, seed=4, mu=0.2)
    c_scene = column_collapse(4096, diameters="lognormal", mu=0.8, aspect=2.0, cic=32)
    c = (c_scene.cfg, c_scene.state, c_scene.radius)
    steps = 120
    batch = SceneBatch([a[0], b[0], c[0]], [a[1], b[1], c[1]], radii=[a[2], b[2], c[2]])
    assert batch.scenes == 3
    assert [r.count for r in batch.ranges] == [3000, 1500, 4096]
    batch.advance(steps)
    for k, (cfg, st, rad) in enumerate((a, b, c)):
        solo = _solo(cfg, st, rad, steps)
        _check_scene(batch, k, solo)
        _check_history(batch, k, solo)
        solo.close()
    batch.close()


def test_batch_picard_fixed_iterations_match_solo():
    scenes = [packed_poly(n=2000, seed=s, mu=0.4, picard=True, tol=0.0) for s in (5, 6)]
    steps = 40
    batch = SceneBatch([s[0] for s in scenes], [s[1] for s in scenes],
                       radii=[s[2] for s in scenes])
    batch.advance(steps)
    for k, (cfg, st, rad) in enumerate(scenes):
        solo = _solo(cfg, st, rad, steps)
        _check_scene(batch, k, solo)
        _check_history(batch, k, solo)
        solo.close()
    batch.close()


def test_batch_no_history_reference_cubes_match_solo():
    cfgs, states = [], []
    for jitter in (0.1, 0.3, 0.5):
        cfg = SimConfig()
        cfg.init_jitter = jitter
        cfg.kernel_timing = False
        st, _ = initial_state(cfg)
        cfgs.append(cfg)
        states.append(st)
    steps = 150
    batch = SceneBatch(cfgs, states)
    batch.advance(steps)
    for k in range(3):
        solo = _solo(cfgs[k], states[k], None, steps)
        _check_scene(batch, k, solo)
        solo.close()
    batch.close()


def test_perturbed_ensemble_members_match_solo_and_diverge():
    base = column_collapse(4096, diameters="uniform", cic=32)
    members = perturbed_members(base, 4, sigma=50e-6, seed=11)
    batch = SceneBatch.from_scenes(members)
    steps = 100
    batch.advance(steps)
    states = batch.scene_states()
    solo = _solo(members[2].cfg, members[2].state, members[2].radius, steps)
    np.testing.assert_array_equal(states[2], solo.get_state())
    solo.close()
    # different seeds give different members
    assert not np.array_equal(states[0], states[1])
    batch.close()


def test_batch_set_dt_reaches_every_scene():
    a = packed_poly(n=1000, seed=8, mu=0.3)
    b = packed_poly(n=800, seed=9, mu=0.6)
    batch = SceneBatch([a[0], b[0]], [a[1], b[1]], radii=[a[2], b[2]])
    batch.advance(10)
    batch.dt = 5e-6
    batch.advance(10)
    for k, (cfg, st, rad) in enumerate((a, b)):
        solo = ParticleDynamics(cfg, state=st, radius=rad)
        solo.advance(10)
        solo.dt = 5e-6
        solo.advance(10)
        np.testing.assert_array_equal(batch.scene_states()[k], solo.get_state())
        solo.close()
    batch.close()


def test_frozen_scene_stays_put_while_the_others_match_solo():
    a = packed_poly(n=1200, seed=12, mu=0.5)
    b = packed_poly(n=900, seed=13, mu=0.3)
    batch = SceneBatch([a[0], b[0]], [a[1], b[1]], radii=[a[2], b[2]])
    batch.advance(20)
    frozen_state = batch.scene_states()[0].copy()
    batch.freeze(0)
    batch.advance(30)
    np.testing.assert_array_equal(batch.scene_states()[0], frozen_state)
    solo = _solo(b[0], b[1], b[2], 50)
    np.testing.assert_array_equal(batch.scene_states()[1], solo.get_state())
    solo.close()
    batch.freeze(0, False)
    batch.advance(1)
    assert not np.array_equal(batch.scene_states()[0], frozen_state)
    batch.close()


def test_per_scene_stability_and_overflow():
    a = packed_poly(n=1000, seed=14, mu=0.5)
    b = packed_poly(n=1000, seed=15, mu=0.5)
    st_b = b[1].copy()
    st_b[0, 3] = 1e4          # one grain thrown out of scene 1's box within a step
    cfg_b = b[0].copy()
    cfg_b.particles_per_cell = 1   # every shared cell counts as an overflow
    batch = SceneBatch([a[0], cfg_b], [a[1], st_b], radii=[a[2], b[2]])
    batch.advance(5)
    assert batch.stability().tolist() == [True, False]
    ov = batch.overflow_counts()
    assert ov[0] == 0 and ov[1] > 0
    assert batch.grid_overflow_count() == ov.sum()
    assert not batch.is_stable()
    batch.close()


def test_chaos_metrics_against_numpy():
    base = column_collapse(2048, diameters="uniform", cic=16)
    members = perturbed_members(base, 3, sigma=50e-6, seed=21)
    batch = SceneBatch.from_scenes(members)
    batch.advance(60)
    got = batch.chaos_metrics(0)
    pos = batch.split(batch.get_positions(), 3)
    grids = batch.scene_density_grids()
    cfg = base.cfg
    nx, ny, nz = cfg.density_grid_size_x, cfg.density_grid_size_y, cfg.density_grid_size_z
    nodes = nx * ny * nz
    idx = np.arange(nodes)
    coords = np.stack([idx // (ny * nz), (idx // nz) % ny, idx % nz])
    m0 = grids[0][:nodes].astype(np.float64)
    com0 = (coords * m0).sum(1) / m0.sum()
    assert got[0].tolist() == [0.0, 0.0, 0.0]
    for k in (1, 2):
        d = pos[k].reshape(-1, 3).astype(np.float64) - pos[0].reshape(-1, 3)
        m = grids[k][:nodes].astype(np.float64)
        want = [np.sqrt((d * d).sum() / d.shape[0]),
                np.sqrt(((m - m0) ** 2).sum() / (m0 ** 2).sum()),
                np.linalg.norm((coords * m).sum(1) / m.sum() - com0)]
        np.testing.assert_allclose(got[k], want, rtol=1e-12, atol=1e-15)
    batch.close()
