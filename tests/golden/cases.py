"""Seeded parity cases shared by the golden-fixture generator and the tests.

Each case is a YAML text in the reference's schema (src/sim_config.cpp) plus an
initial state written in the reference's state-file format (init type "file"), so
the reference's own ParticleDynamics, the oracle and libworld_b200 all start from
the same bytes. Only compat-mode physics appears here (one radius, table masses,
viscous friction): it is all the reference can run.
"""
from __future__ import annotations

import numpy as np

BASE_YAML = """\
simulation:
  dt: {dt}
  collision_grid_size_x: {gx}
  collision_grid_size_y: {gy}
  collision_grid_size_z: {gz}
  particles_per_cell: {ppc}
  threads_per_block: 256
  density_grid_size_x: {dg}
  density_grid_size_y: {dg}
  density_grid_size_z: {dg}
domain:
  x_min: {lo}
  x_max: {hi}
  y_min: {lo}
  y_max: {hi}
  z_min: {lo}
  z_max: {hi}
physics:
  gravity: 9.81
  particle_radius: {radius}
  max_force: {max_force}
  floor_z: {lo}
  ceiling_z: {hi}
  wall_x_min: {lo}
  wall_x_max: {hi}
  wall_y_min: {lo}
  wall_y_max: {hi}
  restitution: {restitution}
  friction: {friction}
materials:
  masses: [0.0, {mass}]
initialization:
  type: file
  state_path: {state_path}
  particle_material: 1
drivers:
  kernel_timing: false
time_integration:
  solver: {solver}
  picard_iterations: {picard}
"""


def packed_state(n: int, radius: float, lo: float, hi: float, spacing_r: float, seed: int,
                 vel_sigma: float, near_walls: bool = False) -> np.ndarray:
    """Jittered simple-cubic packing with spacing spacing_r * radius (below 2 for
    overlaps), random velocities. near_walls pushes the lattice into a corner so the
    wall contacts are exercised too."""
    rng = np.random.default_rng(seed)
    s = spacing_r * radius
    per = int(np.ceil(n ** (1.0 / 3.0)))
    idx = np.stack(np.meshgrid(np.arange(per), np.arange(per), np.arange(per), indexing="ij"),
                   axis=-1).reshape(-1, 3)[:n].astype(np.float64)
    origin = lo + (0.8 * radius if near_walls else 0.5 * (hi - lo) - 0.5 * per * s)
    pos = origin + idx * s + rng.uniform(-0.15 * radius, 0.15 * radius, size=(n, 3))
    vel = rng.normal(0.0, vel_sigma, size=(n, 3))
    return np.concatenate([pos, vel], axis=1).astype(np.float32)


CASES = {
    # contact-free default cube (1000 grains), as the reference's own tests use it
    "cube_default": dict(kind="cube", steps=1),
    # 2197 grains packed with overlaps, random velocities: pair contacts everywhere
    "packed_sie": dict(kind="packed", n=2197, spacing_r=1.92, seed=11, vel_sigma=0.05,
                       solver="semi_implicit_euler", picard=3, steps=1),
    # same packing, backward Euler / Picard with 3 fixed iterations
    "packed_picard": dict(kind="packed", n=2197, spacing_r=1.92, seed=11, vel_sigma=0.05,
                          solver="backward_euler_picard", picard=3, steps=1),
    # packing pressed into a corner: floor and two walls in contact, with friction
    "packed_walls": dict(kind="packed", n=1331, spacing_r=1.95, seed=5, vel_sigma=0.2,
                         solver="semi_implicit_euler", picard=3, steps=1, near_walls=True),
    # restitution 0.6 (the differentiable window's target run): the damping coefficient
    # the library derives from ln e on the host must match the reference's per-contact
    # device logf to the bit
    "packed_e06": dict(kind="packed", n=2197, spacing_r=1.9, seed=17, vel_sigma=0.1,
                       solver="semi_implicit_euler", picard=3, steps=1, restitution=0.6),
}

PACKED_PARAMS = dict(dt=1e-4, gx=50, gy=50, gz=50, ppc=16, dg=16, lo=-0.5, hi=0.5,
                     radius=0.01, max_force=2000.0, restitution=0.3, friction=0.5, mass=0.8)


def case_inputs(name: str, state_path: str) -> tuple[str | None, np.ndarray | None]:
    """(YAML text, initial state) for a case; YAML None means the built-in defaults."""
    c = CASES[name]
    if c["kind"] == "cube":
        return None, None
    p = dict(PACKED_PARAMS)
    p.update({k: c[k] for k in ("restitution", "friction") if k in c})
    state = packed_state(c["n"], p["radius"], p["lo"], p["hi"], c["spacing_r"], c["seed"],
                         c["vel_sigma"], c.get("near_walls", False))
    text = BASE_YAML.format(state_path=state_path, solver=c["solver"], picard=c["picard"], **p)
    return text, state


def write_state(path: str, state: np.ndarray) -> None:
    st = np.ascontiguousarray(state, "<f4").reshape(-1, 6)
    with open(path, "wb") as f:
        f.write(np.int32(st.shape[0]).astype("<i4").tobytes())
        f.write(st.tobytes())


def csr_from_sets(sets: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    offsets = np.zeros(len(sets) + 1, np.int64)
    offsets[1:] = np.cumsum([len(s) for s in sets])
    flat = np.concatenate(sets).astype(np.int32) if sets else np.zeros(0, np.int32)
    return offsets, flat


def sets_from_csr(offsets: np.ndarray, ids: np.ndarray) -> list[np.ndarray]:
    return [np.sort(ids[offsets[i]:offsets[i + 1]]) for i in range(len(offsets) - 1)]
