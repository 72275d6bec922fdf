"""Parity at the workloads' full sizes.

* C0, the 32,768-grain column (uniform diameters, mu = 0.5 with tangential springs and
  history): bit for bit against the oracle over 100 steps from rest, and over 100 steps
  from the collapsing column (12,000 steps in, tens of thousands of live springs).
* C0 in the reference's own physics against the reference's own step (oracle/_ref,
  its CUDA sources built for sm_100a) on the same GPU: per-grain candidate sets equal
  to the reference's, contact flags equal to the oracle's restatement of the reference's
  test, every contact a reference candidate, and state and rhs within 1e-5 after one
  step, at the initial lattice and at the collapsing column.
* C1 exactly as benched (2^20 grains, lognormal diameters, springs and history): bit
  for bit against the oracle over 5 steps from rest and over 5 steps from the settled
  column (30,000 steps in), with the grid searched every step and on Verlet lists with
  the per-lane and the bulk-staged contact kernels and the shared-memory list build.
* C2, the 2^24-grain dense box (int64 offsets, 288 x 288 x 144 cells): 2 steps bit for
  bit against the oracle.
* C3 Set B: the whole 256-scene design batch (9.5 M grains) for 2,000 steps; four
  sampled scenes equal their solo runs bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from cases import sets_from_csr
from conftest import scaled_error
from scale_cases import assert_same_springs, compat_column, transplant
from world_b200 import ParticleDynamics, SceneBatch, load_config
from world_b200.scenes import column_collapse, ensemble_set_b, scene_for

pytestmark = pytest.mark.gpu


def _check_step_exact(sim, orc, steps):
    for _ in range(steps):
        sim.take_step()
        orc.step()
    g = sim.get_state()
    assert np.array_equal(g, orc.state), (
        f"{int((g != orc.state).sum())} floats differ, max {np.abs(g - orc.state).max():.3e}")
    assert np.array_equal(sim.get_rhs(), orc.rhs)
    assert sim.history_overflow_count() == orc.hist_overflow
    return assert_same_springs(sim, orc) if sim.config.history else 0


# ------------------------------------------------------------------ C0 ------------
def test_c0_column_from_rest_bit_exact(oracle_for):
    sc = column_collapse(32768, diameters="uniform", cic=64)
    assert sc.n == 32768 and sc.spec.history
    sim = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
    orc = oracle_for(sc.cfg, sc.state, radius=sc.radius)
    _check_step_exact(sim, orc, 100)
    assert sim.grid_overflow_count() == orc.overflow
    sim.close()


@pytest.mark.parametrize("skin_d", [0.0, 0.15])
def test_c0_collapsing_column_bit_exact(oracle_for, skin_d):
    sc = column_collapse(32768, diameters="uniform", cic=64)
    sc.cfg.neighbor_skin = skin_d * 5e-3
    sim = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
    sim.advance(12000)
    orc = transplant(sim, oracle_for)
    springs = _check_step_exact(sim, orc, 100)
    assert springs > 10000          # the lower column is in contact
    assert sim.compute_total_energy() == pytest.approx(orc.energy(), rel=1e-12)
    sim.close()


@pytest.mark.parametrize("pre_roll", [0, 12000])
def test_c0_sets_and_step_match_reference(tmp_path, oracle_for, pre_roll):
    """The reference searches at the pre-step positions s0 and fills its neighbor rows
    (src/find_neighbors_kernel.cu:119-161); after its step those rows, its rhs f(s0)
    and its state s1 are compared with ours started from the same s0 bytes."""
    from oracle.oracle import ReferenceSim
    if not ReferenceSim.available():
        pytest.fail("oracle/_ref/libref_world.so missing (oracle/build.py builds it)")
    yaml_path, _ = compat_column(tmp_path, 32768, cic=64)
    ref = ReferenceSim(str(yaml_path))
    assert ref.n == 32768
    ref.step(pre_roll)
    s0 = ref.state()
    ref.step(1)
    ref_sets = ref.neighbor_sets()
    ref_s1 = ref.state().reshape(-1, 6)
    ref_rhs = ref.rhs().reshape(-1, 6)
    assert ref.overflow() == 0         # no grain dropped from a full cell
    ref.close()

    cfg = load_config(str(yaml_path))
    sim = ParticleDynamics(cfg, state=s0)
    off, cand, contact = sim.debug_candidates()
    ours = sets_from_csr(off, cand)
    assert len(ours) == len(ref_sets) == 32768
    bad = [k for k in range(32768) if not np.array_equal(ours[k], ref_sets[k])]
    assert not bad, f"{len(bad)} grains' candidate sets differ (first {bad[:5]})"
    o_off, o_cand, o_contact, _ = oracle_for(cfg, s0).candidates()
    assert np.array_equal(off, o_off) and np.array_equal(cand, o_cand)
    assert np.array_equal(contact, o_contact)
    for k in range(32768):
        row = cand[off[k]:off[k + 1]]
        assert np.isin(row[contact[off[k]:off[k + 1]] == 1], ref_sets[k]).all()
    if pre_roll:
        assert contact.sum() > 10000
    sim.take_step()
    s1 = sim.get_state().reshape(-1, 6)
    rhs = sim.get_rhs().reshape(-1, 6)
    assert scaled_error(s1[:, :3], ref_s1[:, :3]) <= 1e-5
    assert scaled_error(s1[:, 3:], ref_s1[:, 3:]) <= 1e-5
    assert scaled_error(rhs[:, 3:], ref_rhs[:, 3:]) <= 1e-5
    sim.close()


# ------------------------------------------------------------------ C1 ------------
C1_MODES = {
    "searched": (0.0, None, False),
    "lists_per_lane": (0.15, (128, 64), False),
    "lists_bulk_staged": (0.15, (256, 1), False),
    "lists_tiled_build": (0.15, (128, 48), True),
}


def _c1_sim(state, radius, mode, springs=None):
    sc = scene_for("collapse_1m_sie_mu05", seed=12345)
    skin_d, kernel, tiled = C1_MODES[mode]
    sc.cfg.neighbor_skin = skin_d * 5e-3
    sim = ParticleDynamics(sc.cfg, state=state, radius=radius)
    if kernel:
        sim.set_contact_kernel(*kernel)
    if tiled:
        sim.set_build_kernel(True)
    if springs is not None:
        sim.set_history(*springs)
    return sim


@pytest.fixture(scope="module")
def c1_settled():
    """The benched column 30,000 steps in (collapsed onto the floor): state, radii and
    springs, reached on Verlet lists (the same bytes as searching every step)."""
    sc = scene_for("collapse_1m_sie_mu05", seed=12345)
    sc.cfg.neighbor_skin = 0.15 * 5e-3
    sim = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
    sim.advance(30000)
    out = (sim.get_state(), sc.radius, sim.get_history())
    sim.close()
    return out


@pytest.mark.parametrize("mode", sorted(C1_MODES))
def test_c1_bench_workload_from_rest_bit_exact(oracle_for, mode):
    sc = scene_for("collapse_1m_sie_mu05", seed=12345)
    assert sc.n == 1 << 20 and sc.spec.history and sc.spec.physics.friction == 0.5
    sim = _c1_sim(sc.state, sc.radius, mode)
    orc = oracle_for(sim.config, sc.state, radius=sc.radius)
    _check_step_exact(sim, orc, 5)
    sim.close()


@pytest.mark.parametrize("mode", sorted(C1_MODES))
def test_c1_settled_column_bit_exact(oracle_for, c1_settled, mode):
    state, radius, springs = c1_settled
    assert int(springs[0].sum()) > 100000
    sim = _c1_sim(state, radius, mode, springs)
    orc = transplant(sim, oracle_for)
    live = _check_step_exact(sim, orc, 5)
    assert live > 100000
    sim.close()


# ------------------------------------------------------------------ C2 ------------
def test_c2_dense_box_two_steps_bit_exact(oracle_for):
    """The dense box starts on a lattice with gaps; 300 steps of its random velocities
    (run by the library) bring it into contact, then 2 steps are checked against the
    oracle from that state and its springs."""
    import psutil
    avail = psutil.virtual_memory().available
    # the oracle's and the library's copies of 24 springs per grain: about 30 GB
    assert avail > 48 << 30, f"{avail / 2**30:.0f} GiB of host memory free; the check needs 48"
    sc = scene_for("dense_16m")
    assert sc.n == 1 << 24
    assert [sc.spec.collision_grid_size_x, sc.spec.collision_grid_size_y,
            sc.spec.collision_grid_size_z] == [288, 288, 144]
    sc.cfg.neighbor_skin = 0.1 * 2 * float(sc.radius[0])
    sim = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
    sim.advance(300)
    orc = transplant(sim, oracle_for)
    live = _check_step_exact(sim, orc, 2)
    assert live > 1 << 20             # springs on a good share of the 2^24 grains
    sim.close()


# ------------------------------------------------------------------ C3 ------------
def test_c3_design_batch_sampled_scenes_match_solo():
    members = ensemble_set_b()
    assert len(members) == 256
    for m in members:
        m.cfg.neighbor_skin = 0.15 * 5e-3
    batch = SceneBatch.from_scenes(members)
    assert batch.n == sum(m.n for m in members) > 9_000_000
    steps = 2000
    batch.advance(steps)
    states = batch.scene_states()
    cnt, part, xi = batch.get_history()
    energies = batch.scene_energies()
    rng = np.random.default_rng(256)
    picks = sorted(set(rng.choice(256, size=4, replace=False).tolist())
                   | {int(np.argmax([m.n for m in members]))})
    for k in picks:
        m = members[k]
        solo = ParticleDynamics(m.cfg, state=m.state, radius=m.radius)
        solo.advance(steps)
        np.testing.assert_array_equal(states[k], solo.get_state())
        r = batch.ranges[k]
        s_cnt, s_part, s_xi = solo.get_history()
        np.testing.assert_array_equal(cnt[r.first:r.first + r.count], s_cnt)
        cap = s_part.size // solo.n
        p = part[r.first * cap:(r.first + r.count) * cap].copy()
        live = (np.arange(p.size) % cap) < np.repeat(s_cnt, cap)
        p[live & (p >= 0)] -= r.first
        np.testing.assert_array_equal(p[live], s_part[live])
        x = xi[3 * r.first * cap:3 * (r.first + r.count) * cap].reshape(-1, 3)
        np.testing.assert_array_equal(x[live], s_xi.reshape(-1, 3)[live])
        assert energies[k] == solo.compute_total_energy()
        solo.close()
    batch.close()
