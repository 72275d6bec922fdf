"""The FP64 restatement used to check the reverse pass (tests/adjoint_ref.py) against
the oracle's FP32 step, and its own frozen-pattern replay. CPU only."""
from __future__ import annotations

import numpy as np

from adjoint_ref import Model, cic, run
from oracle.oracle import OracleSim, params_from_config
from test_gpu_parity import packed_poly
from world_b200.state_io import grain_properties


def model_for(cfg, radius, mass):
    ph = cfg.physics
    return Model(radius=radius.astype(np.float64), mass=mass.astype(np.float64), dt=float(cfg.dt),
                 gravity=float(ph.gravity),
                 wall_lo=np.array([ph.wall_x_min, ph.wall_y_min, ph.floor_z], np.float64),
                 wall_hi=np.array([ph.wall_x_max, ph.wall_y_max, ph.ceiling_z], np.float64),
                 max_force=float(ph.max_force) if ph.max_force > 0 else np.inf,
                 history=bool(cfg.history), kt_fixed=float(ph.tangential_stiffness))


def scene(history, n=400, seed=3):
    cfg, st, rad = packed_poly(n=n, seed=seed, mu=0.5, history=history)
    _, mass = grain_properties(cfg, np.full(n, cfg.particle_material, np.int32), rad)
    return cfg, st, rad, mass


def test_fp64_restatement_follows_the_oracle(_built):
    for history in (True, False):
        cfg, st, rad, mass = scene(history)
        ora = OracleSim(params_from_config(cfg), st, rad, mass)
        model = model_for(cfg, rad, mass)
        ph = cfg.physics
        steps = 30
        ora.step(steps)
        x, v, pat = run(model, st[:, :3], st[:, 3:], ph.friction, ph.restitution,
                        ph.normal_stiffness, steps)
        got = ora.state.reshape(-1, 6)
        assert sum(p.pairs[0].size for p in pat) > 1000      # contacts were exercised
        assert np.abs(got[:, :3] - x).max() < 1e-6
        assert np.abs(got[:, 3:] - v).max() < 1e-3 * np.abs(v).max() + 1e-6


def test_frozen_pattern_replays_the_run():
    cfg, st, rad, mass = scene(True, n=200)
    model = model_for(cfg, rad, mass)
    ph = cfg.physics
    x, v, pat = run(model, st[:, :3], st[:, 3:], ph.friction, ph.restitution, ph.normal_stiffness, 10)
    x2, v2, _ = run(model, st[:, :3], st[:, 3:], ph.friction, ph.restitution, ph.normal_stiffness,
                    10, pattern=pat)
    np.testing.assert_array_equal(x, x2)
    np.testing.assert_array_equal(v, v2)


def test_cic_restatement_conserves_mass_and_momentum():
    rng = np.random.default_rng(0)
    x = rng.uniform(-0.9, 0.9, (50, 3))
    v = rng.normal(size=(50, 3))
    m = rng.uniform(0.5, 2.0, 50)
    g = cic(x, v, m, [-1, -1, -1], [1, 1, 1], (8, 8, 8))
    assert abs(g[0].sum() - m.sum()) < 1e-12
    np.testing.assert_allclose(g[1:].reshape(3, -1).sum(1), (m[:, None] * v).sum(0), rtol=1e-12)
