"""Helpers for the parity tests at the workloads' full sizes.

compat_column(): a column collapse in the reference's own physics (one radius,
material-table mass, viscous friction, max_force = k_n r), written as the reference's
YAML plus state file so that the reference's step (oracle/_ref) and the library load
the same bytes. transplant(): an oracle continuing from a library run's state and
tangential springs, so that a contact-bearing state reached on the GPU in seconds can
be checked step for step on the CPU.
"""
from __future__ import annotations

import numpy as np

from cases import write_state

COMPAT_YAML = """\
simulation:
  dt: 1.0e-5
  collision_grid_size_x: {gx}
  collision_grid_size_y: {gy}
  collision_grid_size_z: {gz}
  particles_per_cell: 8
  threads_per_block: 256
  density_grid_size_x: {cic}
  density_grid_size_y: {cic}
  density_grid_size_z: {cic}
domain:
  x_min: {xlo}
  x_max: {xhi}
  y_min: {xlo}
  y_max: {xhi}
  z_min: 0.0
  z_max: {zhi}
physics:
  gravity: 9.81
  particle_radius: 0.0025
  max_force: 250.0
  floor_z: 0.0
  ceiling_z: {zhi}
  wall_x_min: {xlo}
  wall_x_max: {xhi}
  wall_y_min: {xlo}
  wall_y_max: {xhi}
  restitution: 0.5
  friction: 0.5
materials:
  masses: [0.0, {mass}]
initialization:
  type: file
  state_path: {state_path}
  particle_material: 1
drivers:
  kernel_timing: false
time_integration:
  solver: semi_implicit_euler
  picard_iterations: 3
"""


def compat_column(tmp_path, n: int, cic: int, cell: float | None = None):
    """(yaml path, Scene) of the n-grain column in compat mode: d = 5 mm for every
    grain, mass 2500 kg/m^3 x 4/3 pi r^3 from the material table, mu = 0.5 viscous,
    k_n = 1e5 N/m as max_force = k_n r = 250 N, e = 0.5. The collision grid is
    floor(L / cell) per axis, cell = 1.1 d unless given."""
    from world_b200.scenes import column_collapse
    sc = column_collapse(n, diameters="mono", mu=0.5, history=False, cic=cic)
    dom = sc.spec.domain
    lx = dom.x_max - dom.x_min
    cell = cell or 1.1 * 5e-3
    gx = int(np.floor(lx / cell))
    gz = int(np.floor(dom.z_max / cell))
    mass = 2500.0 * 4.0 / 3.0 * np.pi * 0.0025 ** 3
    state_path = tmp_path / f"compat_{n}.bin"
    write_state(str(state_path), sc.state)
    yaml_path = tmp_path / f"compat_{n}.yaml"
    yaml_path.write_text(COMPAT_YAML.format(
        gx=gx, gy=gx, gz=gz, cic=cic, xlo=repr(-0.5 * lx), xhi=repr(0.5 * lx),
        zhi=repr(float(dom.z_max)), mass=repr(float(np.float32(mass))), state_path=state_path))
    return yaml_path, sc


def transplant(sim, oracle_for):
    """An OracleSim holding `sim`'s current state, grain properties and tangential
    springs (rows by grain id, partners by grain id), with the sim's config."""
    orc = oracle_for(sim.config, sim.get_state(), radius=sim.grain_radius, mass=sim.grain_mass)
    if sim.config.history:
        cnt, part, xi = sim.get_history()
        orc.hcnt[:] = cnt
        orc.hpart[:] = part
        orc.hxi[:] = xi
    return orc


def assert_same_springs(sim, orc):
    cnt, part, xi = sim.get_history()
    np.testing.assert_array_equal(cnt, orc.hcnt)
    cap = part.size // sim.n
    live = (np.arange(part.size) % cap) < np.repeat(cnt, cap)
    np.testing.assert_array_equal(part[live], orc.hpart[live])
    np.testing.assert_array_equal(xi.reshape(-1, 3)[live], orc.hxi.reshape(-1, 3)[live])
    return int(cnt.astype(np.int64).sum())
