"""Verlet lists (simulation.neighbor_skin > 0) against the searched step.

With a skin the grid search runs only when some grain has moved 0.49 skin since the
last list build; contacts are taken from the lists and accumulated in the searched
step's canonical order. States, springs and energies must equal the searched run's
(skin 0, itself bit-identical to the oracle) to the last bit, in graph and in direct
launch mode, for single scenes and batches, including the list-overflow fallback."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import OracleSim, params_from_config
from test_gpu_parity import packed_poly
from world_b200 import ParticleDynamics, SceneBatch, SimConfig
from world_b200.scenes import column_collapse
from world_b200.state_io import grain_properties, initial_state

pytestmark = pytest.mark.gpu


def _pair(cfg, state, radius, steps, skin, timing=False):
    out = []
    for sk in (0.0, skin):
        c = cfg.copy()
        c.neighbor_skin = sk
        c.kernel_timing = timing
        sim = ParticleDynamics(c, state=state, radius=radius)
        sim.advance(steps)
        out.append(sim)
    return out


def _same(a, b):
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    ca, pa, xa = a.get_history()
    cb, pb, xb = b.get_history()
    np.testing.assert_array_equal(ca, cb)
    live = (np.arange(pa.size) % 24) < np.repeat(ca, 24)
    np.testing.assert_array_equal(pa[live], pb[live])
    np.testing.assert_array_equal(xa.reshape(-1, 3)[live], xb.reshape(-1, 3)[live])
    np.testing.assert_array_equal(a.get_rhs(), b.get_rhs())
    assert a.compute_total_energy() == b.compute_total_energy()


@pytest.mark.parametrize("timing", [False, True])
def test_lists_equal_search_every_step_packed_springs(timing):
    cfg, st, rad = packed_poly(n=3000, seed=21, mu=0.5)
    ref, lst = _pair(cfg, st, rad, 200, 0.5e-3, timing)
    _same(ref, lst)
    builds, kernels, mean_len = lst.list_stats()
    assert 1 <= builds < 200 and kernels > 0 and mean_len > 0.5
    assert ref.list_stats()[0] == 0


def test_lists_equal_search_every_step_reference_cube():
    cfg = SimConfig()
    cfg.init_jitter = 0.3
    cfg.kernel_timing = False
    st, _ = initial_state(cfg)
    ref, lst = _pair(cfg, st, None, 300, 2e-3)
    _same(ref, lst)


def test_lists_equal_search_in_a_collapsing_column():
    sc = column_collapse(8192, diameters="lognormal", mu=0.5, cic=32)
    sc.cfg.kernel_timing = False
    ref, lst = _pair(sc.cfg, sc.state, sc.radius, 400, 0.1 * 5e-3)
    _same(ref, lst)
    assert lst.list_stats()[0] < 400


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("skin", [1.5e-3, 2.5e-3])
def test_lists_hold_pairs_two_cells_apart(axis, skin):
    """Cells exactly one grain diameter wide (5 mm): two grains in cells two apart along
    an axis, 5.5 mm between centres, closing at 2 m/s. They are closer than
    r_i + r_j + skin at the build, meet 25 steps later, long before either has moved
    0.49 skin, so the lists must hold the pair although the 27-cell stencil does not
    reach it. The list run must equal the searched one, collision included."""
    cfg = SimConfig()
    L = 0.05
    for ax in "xyz":
        setattr(cfg.domain, f"{ax}_min", -L)
        setattr(cfg.domain, f"{ax}_max", L)
    ph = cfg.physics
    ph.wall_x_min = ph.wall_y_min = ph.floor_z = -L
    ph.wall_x_max = ph.wall_y_max = ph.ceiling_z = L
    ph.gravity = 0.0
    ph.normal_stiffness = 1e5
    ph.max_force = 250.0
    ph.restitution = 0.5
    ph.friction = 0.5
    ph.density = 2500.0
    ph.particle_radius = 2.5e-3
    cfg.history = True
    cfg.collision_grid_size_x = cfg.collision_grid_size_y = cfg.collision_grid_size_z = 20
    cfg.particles_per_cell = 16
    cfg.dt = 1e-5
    cfg.density_grid_size_x = cfg.density_grid_size_y = cfg.density_grid_size_z = 8
    cfg.kernel_timing = False
    state = np.zeros((2, 6), np.float32)
    state[:, :3] = 2.5e-3                      # the middle of cell 10 on the other axes
    state[0, axis], state[1, axis] = -0.3e-3, 5.2e-3   # cells 9 and 11
    state[0, 3 + axis], state[1, 3 + axis] = 1.0, -1.0
    radius = np.full(2, 2.5e-3, np.float32)
    ref, lst = _pair(cfg, state, radius, 100, skin)
    _same(ref, lst)
    v = ref.get_state().reshape(-1, 6)
    assert v[0, 3 + axis] < 0.9 and v[1, 3 + axis] > -0.9     # they did collide
    assert lst.list_stats()[0] < 100


def test_builds_follow_the_displacement_bound():
    """Grains drifting at 0.5 m/s without contacts or gravity: the decision on the
    displacement bound builds every 0.49 skin / (v dt) = 98 steps, as the exact criterion
    does, and reads the build positions only on the steps just before a build."""
    cfg, _, _ = packed_poly(n=512, seed=40)
    cfg.physics.gravity = 0.0
    cfg.kernel_timing = False
    d = 5e-3
    idx = np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij"), -1).reshape(-1, 3)
    state = np.zeros((512, 6), np.float32)
    state[:, :3] = -0.03 + idx * 1.5 * d
    state[:, 3] = 0.5
    radius = np.full(512, 0.5 * d, np.float32)
    ref, lst = _pair(cfg, state, radius, 400, 1e-3)
    np.testing.assert_array_equal(ref.get_state(), lst.get_state())
    builds = lst.list_stats()[0]
    assert builds == 5                      # steps 1, 99, 197, 295, 393 (one either way)
    assert lst.list_exact_count() <= 3 * builds


def test_tiny_skin_and_overflowing_lists_stay_exact():
    cfg, st, rad = packed_poly(n=1500, seed=22, mu=0.3)
    cfg.kernel_timing = False
    # a skin far below a step's motion: a build every step
    ref, lst = _pair(cfg, st, rad, 60, 1e-9)
    _same(ref, lst)
    # a skin of several diameters: lists overflow, the searched path takes over
    ref, lst = _pair(cfg, st, rad, 60, 2e-2)
    _same(ref, lst)


def test_lists_match_the_oracle():
    cfg, st, rad = packed_poly(n=1200, seed=23, mu=0.5)
    cfg.neighbor_skin = 0.4e-3
    cfg.kernel_timing = False
    _, mass = grain_properties(cfg, np.full(st.shape[0], cfg.particle_material, np.int32), rad)
    sim = ParticleDynamics(cfg, state=st, radius=rad)
    ref = OracleSim(params_from_config(cfg), st, rad, mass)
    sim.advance(80)
    ref.step(80)
    np.testing.assert_array_equal(sim.get_state(), ref.state)


def test_set_state_mid_run_rebuilds():
    cfg, st, rad = packed_poly(n=1000, seed=24, mu=0.4)
    ref, lst = _pair(cfg, st, rad, 30, 0.5e-3)
    mid = ref.get_state().reshape(-1, 6).copy()
    mid[:, 2] += 1e-4                     # every grain lifted: old lists are stale
    ref.set_state(mid)
    lst.set_state(mid)
    ref.advance(40)
    lst.advance(40)
    _same(ref, lst)


def test_batch_with_lists_equals_searched_batch():
    a = packed_poly(n=1200, seed=25, mu=0.5)
    b = packed_poly(n=900, seed=26, mu=0.2)
    sims = []
    for skin in (0.0, 0.5e-3):
        cfgs = []
        for c in (a[0], b[0]):
            cc = c.copy()
            cc.neighbor_skin = skin
            cc.kernel_timing = False
            cfgs.append(cc)
        sb = SceneBatch(cfgs, [a[1], b[1]], radii=[a[2], b[2]])
        sb.advance(150)
        sims.append(sb)
    _same(*sims)


def test_skin_switch_mid_run_stays_exact():
    cfg, st, rad = packed_poly(n=1500, seed=27, mu=0.5)
    cfg.kernel_timing = False
    ref = ParticleDynamics(cfg, state=st, radius=rad)
    sw = ParticleDynamics(cfg, state=st, radius=rad)
    ref.advance(90)
    sw.advance(30)
    sw.set_neighbor_skin(0.5e-3)
    sw.advance(30)
    sw.set_neighbor_skin(0.0)
    sw.advance(15)
    sw.set_neighbor_skin(1e-3)
    sw.advance(15)
    _same(ref, sw)


def test_autotune_restores_the_state_and_caches(tmp_path):
    sc = column_collapse(8192, diameters="lognormal", mu=0.5, cic=32)
    sc.cfg.kernel_timing = False
    ref = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
    tuned = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
    ref.advance(20)
    tuned.advance(20)
    before = tuned.get_state()
    t0 = tuned.time
    cache = tmp_path / "tune.txt"
    skin, block = tuned.autotune(steps=20, cache=str(cache))
    assert block in (128, 256) and skin >= 0.0
    np.testing.assert_array_equal(tuned.get_state(), before)
    assert tuned.time == t0
    ref.advance(50)
    tuned.advance(50)
    _same(ref, tuned)
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and lines[0].startswith("n=8192,")
    other = ParticleDynamics(sc.cfg, state=sc.state, radius=sc.radius)
    assert other.autotune(steps=20, cache=str(cache)) == (np.float32(skin), block)
    assert len(cache.read_text().splitlines()) == 1


@pytest.mark.parametrize("variant,block", [(0, 256), (64, 128), (48, 64), (1, 256), (2, 256)])
def test_every_contact_kernel_variant_is_exact(variant, block):
    cfg, st, rad = packed_poly(n=2500, seed=28, mu=0.5)
    cfg.kernel_timing = False
    ref = ParticleDynamics(cfg, state=st, radius=rad)
    c = cfg.copy()
    c.neighbor_skin = 0.5e-3
    var = ParticleDynamics(c, state=st, radius=rad)
    var.set_contact_kernel(block, variant)
    ref.advance(150)
    var.advance(150)
    _same(ref, var)
    # viscous friction (no springs) and a batch through the same kernel
    cfg2, st2, rad2 = packed_poly(n=1500, seed=29, mu=0.5, history=False)
    cfg2.kernel_timing = False
    ref2 = ParticleDynamics(cfg2, state=st2, radius=rad2)
    c2 = cfg2.copy()
    c2.neighbor_skin = 0.5e-3
    var2 = ParticleDynamics(c2, state=st2, radius=rad2)
    var2.set_contact_kernel(block, variant)
    ref2.advance(120)
    var2.advance(120)
    _same(ref2, var2)
    sb = []
    for skin in (0.0, 0.5e-3):
        cfgs = []
        for cc in (cfg, cfg2.copy()):
            x = cc.copy()
            x.history = True
            x.neighbor_skin = skin
            cfgs.append(x)
        b = SceneBatch(cfgs, [st, st2], radii=[rad, rad2])
        if skin:
            b.set_contact_kernel(block, variant)
        b.advance(100)
        sb.append(b)
    _same(*sb)


def test_builds_are_launched_from_the_device():
    """In a graph-launched list step the build is not a conditional node: the step graph
    holds the contact kernel and a one-thread kernel that tail-launches the build's
    device graphs (search head, then the mover or radix path) when the contact kernel
    decided a build. Builds happen, and the run equals the searched one."""
    cfg, st, rad = packed_poly(n=2500, seed=32, mu=0.5)
    cfg.kernel_timing = False
    ref = ParticleDynamics(cfg, state=st, radius=rad)
    c = cfg.copy()
    c.neighbor_skin = 0.5e-3
    lst = ParticleDynamics(c, state=st, radius=rad)
    ref.advance(200)
    lst.advance(200)
    _same(ref, lst)
    builds, kernels_each, _ = lst.list_stats()
    assert lst.kernels_per_step() == 2            # the contact kernel and the launcher
    assert kernels_each == 6
    assert 2 <= builds < 200


def test_contact_kernel_switches_mid_run():
    """Switching the list contact kernel between steps (per-lane at 48 and 64
    registers, cooperative, bulk-staged, and back) leaves the run equal to the searched
    one."""
    cfg, st, rad = packed_poly(n=2500, seed=31, mu=0.5)
    cfg.kernel_timing = False
    ref = ParticleDynamics(cfg, state=st, radius=rad)
    c = cfg.copy()
    c.neighbor_skin = 0.5e-3
    var = ParticleDynamics(c, state=st, radius=rad)
    for block, variant in ((128, 48), (256, 0), (128, 64), (256, 1), (256, 0), (128, 48)):
        var.set_contact_kernel(block, variant)
        var.advance(40)
    ref.advance(240)
    _same(ref, var)


def test_bulk_staged_kernel_over_many_tiles():
    """2^20 grains: every warp of the persistent bulk-staged kernel runs several tiles
    (each stage refilled, its barrier phase flipping), and the state stays the searched
    run's."""
    sc = column_collapse(1 << 20, diameters="lognormal", mu=0.5, cic=32)
    sc.cfg.kernel_timing = False
    out = []
    for skin, variant in ((0.0, None), (0.5e-3, 1)):
        c = sc.cfg.copy()
        c.neighbor_skin = skin
        sim = ParticleDynamics(c, state=sc.state, radius=sc.radius)
        if variant is not None:
            sim.set_contact_kernel(256, variant)
            assert sim.tuning()["contact_variant"].startswith("bulk-staged")
        sim.advance(30)
        out.append(sim)
    _same(*out)


def test_dense_contacts_cooperative_kernel_matches_oracle():
    """Many contacts per warp (several queue flushes) through the cooperative kernel."""
    cfg, st, rad = packed_poly(n=3000, seed=30, mu=0.6)
    cfg.neighbor_skin = 0.3e-3
    cfg.kernel_timing = False
    cfg.physics.max_force = 50.0      # clamped contacts too
    _, mass = grain_properties(cfg, np.full(st.shape[0], cfg.particle_material, np.int32), rad)
    sim = ParticleDynamics(cfg, state=st, radius=rad)
    sim.set_contact_kernel(256, 0)
    ref = OracleSim(params_from_config(cfg), st, rad, mass)
    sim.advance(60)
    ref.step(60)
    np.testing.assert_array_equal(sim.get_state(), ref.state)


@pytest.mark.parametrize("timing", [False, True])
def test_picard_on_lists_equals_picard_with_search(timing):
    # tolerance-terminated iterations with springs
    cfg, st, rad = packed_poly(n=2500, seed=31, mu=0.5, picard=True, tol=1e-9)
    ref, lst = _pair(cfg, st, rad, 80, 0.5e-3, timing)
    _same(ref, lst)
    assert ref.picard_stats() == lst.picard_stats()
    # fixed iteration count, viscous friction
    cfg2, st2, rad2 = packed_poly(n=2000, seed=32, mu=0.4, history=False, picard=True, tol=0.0)
    ref2, lst2 = _pair(cfg2, st2, rad2, 60, 0.5e-3, timing)
    _same(ref2, lst2)


def test_picard_redo_when_iterates_leave_the_lists():
    """A skin so small that iterates leave it every step: each step is redone with the
    per-iteration search, and the results stay exact."""
    cfg, st, rad = packed_poly(n=1500, seed=33, mu=0.5, picard=True, tol=1e-9)
    cfg.kernel_timing = False
    ref, lst = _pair(cfg, st, rad, 40, 1e-9)
    _same(ref, lst)
    assert lst.picard_counts()[1] > 0 and ref.picard_counts()[1] == 0
    # the redone steps run their iterations twice (lists, then search)
    assert lst.picard_counts()[0] > ref.picard_counts()[0]


def test_batched_picard_on_lists():
    scenes = [packed_poly(n=1200, seed=s, mu=0.4, picard=True, tol=0.0) for s in (34, 35)]
    sims = []
    for skin in (0.0, 0.5e-3):
        cfgs = []
        for c in (scenes[0][0], scenes[1][0]):
            cc = c.copy()
            cc.neighbor_skin = skin
            cc.kernel_timing = False
            cfgs.append(cc)
        b = SceneBatch(cfgs, [sc[1] for sc in scenes], radii=[sc[2] for sc in scenes])
        b.advance(50)
        sims.append(b)
    _same(*sims)


def test_bulk_staged_wait_runs_out_and_the_handle_recovers():
    """The bulk-staged kernel's bounded wait: a stage made to expect bytes that no copy
    delivers (wd_debug_stage_wait) runs out after 2 ms; the next synchronizing call
    reports it once, and after a state restore the handle steps as a fresh one does."""
    from world_b200 import WorldError
    from world_b200._lib import check, lib
    cfg, st, rad = packed_poly(n=3000, seed=21, mu=0.5)
    cfg.neighbor_skin = 0.5e-3
    cfg.kernel_timing = False
    sim = ParticleDynamics(cfg, state=st, radius=rad)
    sim.set_contact_kernel(256, 1)
    sim.advance(10)
    saved, springs = sim.get_state(), sim.get_history()
    check(lib.wd_debug_stage_wait(sim.handle, 1, 2000))
    sim.take_step()
    with pytest.raises(WorldError, match="wait limit"):
        sim.synchronize()
    sim.synchronize()                       # reported once; the context is usable
    check(lib.wd_debug_stage_wait(sim.handle, 0, 0))
    sim.set_state(saved)
    sim.set_history(*springs)
    sim.advance(20)
    fresh = ParticleDynamics(cfg, state=saved, radius=rad)
    fresh.set_contact_kernel(256, 1)
    fresh.set_history(*springs)
    fresh.advance(20)
    _same(sim, fresh)
    sim.close()
    fresh.close()
