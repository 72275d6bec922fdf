"""Scenes and the CPU stand-in stepper for the slab decomposition tests."""
from __future__ import annotations

import numpy as np

from test_gpu_parity import packed_poly

HIST_CAP = 24


def sheared_pack(n=3000, seed=21):
    """packed_poly with x velocities of +-2 m/s (half each way, by z layer) and dt 2e-5:
    over 80 steps grains travel 3 mm of a 7 mm cell, so many cross the slab cut."""
    cfg, st, rad = packed_poly(n=n, seed=seed, mu=0.5, history=True)
    rng = np.random.default_rng(seed)
    st = st.copy()
    st[:, 3] = np.where(st[:, 2] > np.median(st[:, 2]), 2.0, -2.0) + rng.normal(0, 0.1, n)
    cfg.dt = 2e-5
    return cfg, st, rad


class OracleStepper:
    """The oracle as the local step: a CPU stand-in for libworld_b200 in host tests of
    the decomposition (partition, exchange, id and spring remapping)."""

    def __init__(self, cfg):
        self.cfg = cfg

    def step(self, gid, state, radius, mass, rows):
        from oracle.oracle import OracleSim, params_from_config
        sim = OracleSim(params_from_config(self.cfg), state, radius, mass)
        if rows is not None:
            sim.hcnt[:] = rows[0]
            sim.hpart[:] = rows[1]
            sim.hxi[:] = rows[2]
        sim.step()
        out_rows = (sim.hcnt.copy(), sim.hpart.copy(), sim.hxi.copy()) if rows is not None else None
        return sim.state.reshape(-1, 6).copy(), out_rows

    def grain_energies(self, *a):
        raise NotImplementedError("the oracle has no per-grain energies")
