"""Batched scenes on the host: argument checks of wd_create_batch (they run before
any device call) and the ensemble / design generators."""
from __future__ import annotations

import numpy as np
import pytest

from world_b200 import SceneBatch, WorldError
from world_b200.scenes import column_collapse, ensemble_set_a, ensemble_set_b, perturbed_members


def _two(n0=512, n1=600):
    a = column_collapse(n0, cic=16)
    b = column_collapse(n1, cic=16, seed=4)
    return a, b


def test_scenes_must_share_dt():
    a, b = _two()
    b.cfg.dt = 2e-5
    with pytest.raises(WorldError, match="must share"):
        SceneBatch.from_scenes([a, b])


def test_scenes_must_share_history_and_integrator():
    a, b = _two()
    b.cfg.history = False
    with pytest.raises(WorldError, match="must share"):
        SceneBatch.from_scenes([a, b])
    a, b = _two()
    b.cfg.time_integrator = "backward_euler_picard"
    with pytest.raises(WorldError, match="must share"):
        SceneBatch.from_scenes([a, b])


def test_batch_picard_needs_fixed_iterations():
    a, b = _two()
    for s in (a, b):
        s.cfg.time_integrator = "backward_euler_picard"
        s.cfg.picard_tolerance = 1e-6
    with pytest.raises(WorldError, match="fixed"):
        SceneBatch.from_scenes([a, b])


def test_batch_argument_shapes():
    a, b = _two()
    with pytest.raises(ValueError):
        SceneBatch([a.cfg, b.cfg], [a.state])
    with pytest.raises(ValueError):
        SceneBatch([a.cfg, b.cfg], [a.state, b.state], radii=[a.radius, a.radius])
    with pytest.raises(ValueError):
        SceneBatch([], [])


def test_bad_grid_in_one_scene_is_reported():
    a, b = _two()
    b.cfg.collision_grid_size_y = 0
    with pytest.raises(WorldError, match="grid sizes"):
        SceneBatch.from_scenes([a, b])


def test_perturbed_members_are_seeded_gaussian():
    base = column_collapse(2048, cic=16)
    m1 = perturbed_members(base, 3, sigma=50e-6, seed=5)
    m2 = perturbed_members(base, 3, sigma=50e-6, seed=5)
    for x, y in zip(m1, m2):
        np.testing.assert_array_equal(x.state, y.state)
    d = (m1[0].state[:, :3].astype(np.float64) - base.state[:, :3])
    assert abs(d.std() - 50e-6) < 5e-6
    assert abs(d.mean()) < 5e-6
    assert not np.array_equal(m1[0].state, m1[1].state)
    np.testing.assert_array_equal(m1[0].state[:, 3:], base.state[:, 3:])


def test_ensemble_sets_have_their_sizes():
    a = ensemble_set_a(members=4)
    assert len(a) == 4 and all(s.n == 32768 for s in a)
    b = ensemble_set_b(scenes=32)
    ns = np.array([s.n for s in b])
    assert ns.min() >= 4096 and ns.max() <= 131072
    mus = np.array([s.cfg.physics.friction for s in b])
    assert mus.min() >= 0.0 and mus.max() <= 0.8
    assert len({s.cfg.dt for s in b}) == 1
    assert len({s.cfg.history for s in b}) == 1
