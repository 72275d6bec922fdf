"""The batched dataset and chaos drivers against the reference's sequential
algorithm, run here through single-scene ParticleDynamics objects.

The sequential loops below restate src/dataset.cpp:186-224 and src/chaos.cpp:120-222:
one simulation per design row (or ensemble member), stepped checkpoint by
checkpoint, polled for overflow and stability at every checkpoint, its grid written
or zero-filled. The drivers run the same rows as scenes of one batch (several
batches here, to cover the batch seams), so grids, statuses, final times and
deposited masses must match exactly; the chaos measures are FP64 sums in another
order: relative 1e-12 before the CSV's 9 significant digits.
"""
from __future__ import annotations

import csv
import os

import numpy as np
import pytest

from driver_cases import DESIGN_CSV, run_driver, write_blob
from world_b200 import ParticleDynamics, dataset_io, load_config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _drivers(_built):
    import importlib.util
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wb_build", os.path.join(ROOT, "world_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build_drivers()


def _row_config(base, names, row):
    c = base.copy()
    for name, v in zip(names, row):
        if name == "throw_vx":
            c.init_vx0 = v
        elif name == "throw_vy":
            c.init_vy0 = v
        elif name == "throw_vz":
            c.init_vz0 = v
        elif name == "release_z":
            c.init_z0 = v
        elif name == "grain_mass":
            c.masses = [c.masses[0]] + [v] * (len(c.masses) - 1)
        elif name == "restitution":
            c.physics.restitution = v
        elif name == "friction":
            c.physics.friction = v
    return c


def _sequential_dataset(base, names, rows):
    K = base.dataset_checkpoints
    out = []
    for row in rows:
        cfg = _row_config(base, names, row)
        sim = ParticleDynamics(cfg)
        spc = max(1, int(np.float32(base.dataset_sim_time) /
                         (np.float32(K) * np.float32(cfg.dt)) + np.float32(0.5)))
        diverged, overflow, deposited, grids = False, 0, 0.0, []
        for k in range(K):
            if not diverged:
                sim.advance(spc)
                overflow = sim.grid_overflow_count()
                if overflow > 0 or not sim.is_stable():
                    diverged = True
            if diverged:
                grids.append(np.zeros_like(sim.host_density_grid))
                continue
            sim.compute_density_grid()
            grids.append(sim.host_density_grid.copy())
            if k == K - 1:
                mass = sim.host_density_grid[:sim.density_grid_nodes()].astype(np.float64)
                deposited = float(np.cumsum(mass)[-1])
        out.append(dict(grids=np.stack(grids), status="diverged" if diverged else "ok",
                        time=sim.time, overflow=overflow, deposited=deposited, n=sim.n))
        sim.close()
    return out


def test_dataset_driver_matches_sequential_rollouts(tmp_path):
    cfg_path = write_blob(tmp_path / "blob.yaml", sim_time=0.05, checkpoints=5)
    (tmp_path / "design.csv").write_text(DESIGN_CSV)
    r = run_driver("dataset", [cfg_path, tmp_path / "design.csv", tmp_path / "out", "--batch", 2],
                   tmp_path)
    assert r.returncode == 0, r.stderr
    assert "(4 ok, 1 diverged)" in r.stdout
    d = dataset_io.load(str(tmp_path / "out"))
    base = load_config(cfg_path)
    names = d.parameter_names
    assert names == ["throw_vx", "throw_vz", "release_z", "grain_mass", "restitution", "friction"]
    np.testing.assert_allclose(d.checkpoint_times, np.float32(0.05) * np.arange(1, 6, dtype=np.float32) / np.float32(5))
    seq = _sequential_dataset(base, names, d.parameters.astype(np.float32))
    assert d.grids.shape == (5, 5, 4, 8, 8, 4)
    for i, s in enumerate(seq):
        np.testing.assert_array_equal(d.grids[i].reshape(5, -1), s["grids"])
        assert d.status[i] == s["status"]
        assert d.final_time[i] == float(f"{s['time']:.9g}")
        assert d.overflow_cells[i] == s["overflow"]
        assert d.deposited_mass[i] == float(f"{s['deposited']:.9g}")
    assert d.status[2] == "diverged"
    assert not d.grids[2, -1].any()
    # grains are conserved: deposited mass = n m for the rows that stayed in the box
    n = seq[0]["n"]
    for i in (0, 1, 3, 4):
        assert abs(d.deposited_mass[i] - n * d.parameters[i, 3]) < 1e-4 * n * d.parameters[i, 3]


def test_chaos_driver_matches_sequential_members(tmp_path):
    cfg_path = write_blob(tmp_path / "ens.yaml", sim_time=0.04, checkpoints=4,
                          extra="  perturbation: 0.05\n")
    members = 4
    r = run_driver("chaos", [cfg_path, members, "--batch", 3], tmp_path)
    assert r.returncode == 0, r.stderr
    base = load_config(cfg_path)
    K = base.dataset_checkpoints
    spc = max(1, int(np.float32(base.dataset_sim_time) / (np.float32(K) * np.float32(base.dt)) + np.float32(0.5)))
    ny, nz = base.density_grid_size_y, base.density_grid_size_z
    nodes = base.density_grid_size_x * ny * nz
    idx = np.arange(nodes)
    ix, iy, iz = idx // (ny * nz), (idx // nz) % ny, idx % nz

    def run(cfg):
        sim = ParticleDynamics(cfg)
        pos, fields = [], []
        for _ in range(K):
            sim.advance(spc)
            pos.append(sim.get_positions().astype(np.float64))
            sim.compute_density_grid()
            fields.append(sim.host_density_grid[:nodes].astype(np.float64))
        sim.close()
        return pos, fields

    ref_cfg = base.copy()
    ref_cfg.init_perturbation = 0.0
    ref_pos, ref_fields = run(ref_cfg)

    def com(m):
        t = m.sum()
        return np.array([(m * ix).sum(), (m * iy).sum(), (m * iz).sum()]) / t if t > 0 else np.zeros(3)

    with open(tmp_path / "chaos" / "divergence.csv", newline="") as f:
        rows = list(csv.reader(f))
    assert rows[0] == ["member", "checkpoint", "time", "grain_rms_displacement",
                       "field_relative_difference", "com_displacement"]
    body = rows[1:]
    assert len(body) == (members - 1) * K
    finals = [ref_fields[-1]]
    for m in range(1, members):
        cfg = base.copy()
        cfg.init_perturbation_seed = 1000 + m
        pos, fields = run(cfg)
        finals.append(fields[-1])
        for k in range(K):
            row = body[(m - 1) * K + k]
            assert int(row[0]) == m and int(row[1]) == k
            d = pos[k].reshape(-1, 3) - ref_pos[k].reshape(-1, 3)
            rms = np.sqrt((d * d).sum() / d.shape[0])
            diff = fields[k] - ref_fields[k]
            fr = np.sqrt((diff * diff).sum() / (ref_fields[k] ** 2).sum())
            cd = np.linalg.norm(com(fields[k]) - com(ref_fields[k]))
            for got, want in zip(map(float, row[3:6]), (rms, fr, cd)):
                assert got == pytest.approx(want, rel=1e-7, abs=1e-12)
            assert rms > 0.0
    ff = dataset_io.load_final_fields(str(tmp_path / "chaos" / "final_fields.bin"))
    assert ff.shape == (members, nodes)
    for m in range(members):
        np.testing.assert_array_equal(ff[m], finals[m].astype(np.float32))
