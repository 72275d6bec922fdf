"""Small inputs for the dataset and chaos drivers (shared by the CPU and GPU tests)."""
from __future__ import annotations

import os
import subprocess

from conftest import ROOT

BIN = os.path.join(ROOT, "world_b200", "bin")

# A 216-grain (6^3) jittered blob thrown in a walled 2 x 2 x 1.4 m box: the reference's
# dataset base config (dataset/blob_throw.yaml) scaled down to run in a second.
BLOB_YAML = """\
simulation:
  dt: 0.0001
  collision_grid_size_x: 100
  collision_grid_size_y: 100
  collision_grid_size_z: 70
  particles_per_cell: 8
  density_grid_size_x: 8
  density_grid_size_y: 8
  density_grid_size_z: 4
domain:
  x_min: -1.0
  x_max:  1.0
  y_min: -1.0
  y_max:  1.0
  z_min: -1.0
  z_max:  0.4
physics:
  gravity: 9.81
  particle_radius: 0.01
  max_force: 2000.0
  floor_z:    -1.0
  ceiling_z:   0.4
  wall_x_min: -1.0
  wall_x_max:  1.0
  wall_y_min: -1.0
  wall_y_max:  1.0
  restitution: 0.3
  friction: 0.5
materials:
  masses: [0.0, 0.08]
initialization:
  type: cube
  x0: -0.06
  y0: -0.06
  z0: 0.0
  cube_length_x: 0.12
  cube_length_y: 0.12
  cube_length_z: 0.12
  jitter: 0.25
  seed: 12345
  particle_material: 1
{extra}
dataset:
  sim_time: {sim_time}
  checkpoints: {checkpoints}
"""

# throw_vx = 500 m/s crosses the x wall faster than the clamped wall force can stop
# it, so that row leaves the domain and is reported diverged.
DESIGN_CSV = (
    "throw_vx,throw_vz,release_z,grain_mass,restitution,friction\r\n"
    "0.5,1.0,0.0,0.08,0.3,0.5\r\n"
    "-1.0,0.0,-0.2,0.05,0.5,0.2\r\n"
    "500.0,0.0,0.0,0.08,0.3,0.5\r\n"
    "0.0,-2.0,0.2,0.12,0.1,0.8\r\n"
    "2.0,0.5,-0.5,0.02,0.6,0.0\r\n"
)


def write_blob(path, sim_time=0.05, checkpoints=5, extra=""):
    with open(path, "w") as f:
        f.write(BLOB_YAML.format(sim_time=sim_time, checkpoints=checkpoints, extra=extra))
    return str(path)


def run_driver(name, args, cwd, timeout=600):
    return subprocess.run([os.path.join(BIN, name)] + [str(a) for a in args], cwd=str(cwd),
                          capture_output=True, text=True, timeout=timeout)
