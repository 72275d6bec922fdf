"""Seeded synthetic scenes for the benchmark workloads.

No dataset ships with the reference, so these generators stand in for its runs, with
the shapes, sizes and value distributions of the workloads they name:

* column_collapse(n, ...): granular column collapse. Grains on a simple-cubic lattice
  inside a cylinder of radius R and height 4R, centred in a walled box; the lattice
  spacing is the smallest one whose first n sites (ordered by z, then y, then x) all
  fit; each site is jittered uniformly by +-0.05 d per axis. At n = 32,768 and
  d = 5 mm the box is 1.0 x 1.0 x 0.5 m and R = 0.1 m; larger n scales R and the box
  by (n / 32768)^(1/3). Diameters: "uniform" in [0.9 d, 1.1 d], "lognormal" with
  arithmetic mean d and log-sigma 0.15 clipped to [0.7 d, 1.4 d], or "mono".
* dense_box(n, ...): grains at volume fraction 0.55 in a 2 x 2 x 1 m box on a
  jittered body-centred-cubic lattice (simple cubic tops out at 0.524), velocities
  N(0, 0.5 m/s) per component.

Each returns a Scene: state[n, 6], radius[n] and the configuration as a ConfigSpec
(plain values under SimConfig's member names); `Scene.cfg` is the library's SimConfig
built from it on first use. Masses come from physics.density (2500 kg/m^3), as
grain_properties() states. The collision cell is the larger of 1.1 d and the largest
contact distance (2 r_max), so the 27-cell stencil sees every contact.

This module needs numpy only: it does not load libworld_b200.so until `Scene.cfg` is
read, so CPU-side tools (the oracle's timed baseline) can build the same scenes.
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass, field
from types import SimpleNamespace
from typing import Any

import numpy as np

D_REF = 5e-3          # mean diameter d (m)
N_REF = 32768         # grains of the 1.0 x 1.0 x 0.5 m reference column


class ConfigSpec:
    """The SimConfig members the scene generators set, as plain Python values under
    the same names (`spec.domain.x_min`, `spec.physics.friction`, `spec.dt`, ...);
    every other member keeps the reference's default (src/sim_config.h:68-199).
    `to_config()` gives the library's SimConfig with these values."""

    _TOP = ("dt", "collision_grid_size_x", "collision_grid_size_y", "collision_grid_size_z",
            "particles_per_cell", "density_grid_size_x", "density_grid_size_y",
            "density_grid_size_z", "history", "neighbor_skin", "time_integrator",
            "picard_iterations", "picard_tolerance", "kernel_timing", "particle_material",
            "masses")
    _DOMAIN = ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max")
    _PHYSICS = ("gravity", "particle_radius", "max_force", "floor_z", "ceiling_z",
                "wall_x_min", "wall_x_max", "wall_y_min", "wall_y_max", "restitution",
                "friction", "normal_stiffness", "tangential_stiffness", "density")

    def __init__(self) -> None:
        # reference defaults for the members the generators leave alone
        self.particle_material = 1
        self.masses = [0.0, 0.04]
        self.neighbor_skin = 0.0
        self.kernel_timing = False
        self.domain = SimpleNamespace(**{k: 0.0 for k in self._DOMAIN})
        self.physics = SimpleNamespace(**{k: 0.0 for k in self._PHYSICS})

    def copy(self) -> "ConfigSpec":
        return copy.deepcopy(self)

    def to_config(self):
        from .config import SimConfig   # loads the library
        cfg = SimConfig()
        for k in self._TOP:
            setattr(cfg, k, getattr(self, k))
        for k in self._DOMAIN:
            setattr(cfg.domain, k, getattr(self.domain, k))
        for k in self._PHYSICS:
            setattr(cfg.physics, k, getattr(self.physics, k))
        return cfg


@dataclass
class Scene:
    spec: ConfigSpec
    state: np.ndarray    # (n, 6) float32
    radius: np.ndarray   # (n,) float32
    name: str
    _cfg: Any = field(default=None, repr=False)

    @property
    def n(self) -> int:
        return int(self.state.shape[0])

    @property
    def cfg(self):
        """The library's SimConfig for this scene (built once; changes made to it stay
        with the scene)."""
        if self._cfg is None:
            self._cfg = self.spec.to_config()
        return self._cfg


def grain_properties(cfg, material: np.ndarray,
                     radius: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Per-grain (radius, mass) the library derives when none are given: the global
    particle_radius, and mass from physics.density (4/3 pi r^3 rho, evaluated in
    double and rounded once to float) when it is set, else the materials.masses table.
    `cfg` is a SimConfig or a ConfigSpec."""
    n = material.size
    r = np.full(n, np.float32(cfg.physics.particle_radius), np.float32) if radius is None \
        else np.asarray(radius, np.float32)
    rho = cfg.physics.density
    if rho > 0:
        rd = r.astype(np.float64)
        m = (np.float64(np.float32(rho)) * 4.0 / 3.0 * np.pi * rd * rd * rd).astype(np.float32)
    else:
        table = np.asarray(cfg.masses, np.float32)
        m = table[material]
    return r, m


def _diameters(rng: np.random.Generator, n: int, d: float, kind: str) -> np.ndarray:
    if kind == "mono":
        return np.full(n, d, np.float64)
    if kind == "uniform":
        return rng.uniform(0.9 * d, 1.1 * d, n)
    if kind == "lognormal":
        sigma = 0.15
        mu = math.log(d) - 0.5 * sigma * sigma
        return np.clip(rng.lognormal(mu, sigma, n), 0.7 * d, 1.4 * d)
    raise ValueError(f"unknown diameter distribution '{kind}'")


def _cylinder_sites(n: int, spacing: float, radius_xy: float, z0: float) -> np.ndarray | None:
    k = int(math.floor(radius_xy / spacing))
    ax = np.arange(-k, k + 1, dtype=np.float64) * spacing
    yy, xx = np.meshgrid(ax, ax, indexing="ij")          # rows: y, cols: x
    inside = (xx * xx + yy * yy) <= radius_xy * radius_xy
    layer = np.stack([xx[inside], yy[inside]], axis=1)    # (y, x) order within a layer
    per_layer = layer.shape[0]
    if per_layer == 0:
        return None
    layers = -(-n // per_layer)
    z = z0 + np.arange(layers, dtype=np.float64) * spacing
    sites = np.concatenate([np.column_stack([layer, np.full(per_layer, zz)]) for zz in z])
    return sites[:n]


def _apply_common(cfg: ConfigSpec, box: tuple[float, float, float], d_max: float, d_mean: float,
                  *, mu: float, restitution: float, k_n: float, density: float, dt: float,
                  history: bool, integrator: str, picard_iterations: int, picard_tol: float,
                  cic: int, cell_factor: float = 1.1) -> None:
    lx, ly, lz = box
    cfg.domain.x_min, cfg.domain.x_max = -0.5 * lx, 0.5 * lx
    cfg.domain.y_min, cfg.domain.y_max = -0.5 * ly, 0.5 * ly
    cfg.domain.z_min, cfg.domain.z_max = 0.0, lz
    ph = cfg.physics
    ph.wall_x_min, ph.wall_x_max = -0.5 * lx, 0.5 * lx
    ph.wall_y_min, ph.wall_y_max = -0.5 * ly, 0.5 * ly
    ph.floor_z, ph.ceiling_z = 0.0, lz
    ph.gravity = 9.81
    ph.particle_radius = 0.5 * d_mean
    ph.normal_stiffness = k_n
    ph.max_force = k_n * 0.5 * d_mean          # clamp at one mean radius of overlap
    ph.restitution = restitution
    ph.friction = mu
    ph.density = density
    cfg.history = history and mu > 0
    cfg.dt = dt
    cell = max(cell_factor * d_mean, d_max)
    cfg.collision_grid_size_x = max(1, int(math.floor(lx / cell)))
    cfg.collision_grid_size_y = max(1, int(math.floor(ly / cell)))
    cfg.collision_grid_size_z = max(1, int(math.floor(lz / cell)))
    cfg.particles_per_cell = 16
    cfg.density_grid_size_x = cic
    cfg.density_grid_size_y = cic
    cfg.density_grid_size_z = cic
    cfg.time_integrator = integrator
    cfg.picard_iterations = picard_iterations
    cfg.picard_tolerance = picard_tol
    cfg.kernel_timing = False


def column_collapse(n: int = N_REF, *, diameters: str = "uniform", seed: int = 12345,
                    mu: float = 0.5, restitution: float = 0.5, k_n: float = 1e5,
                    density: float = 2500.0, dt: float = 1e-5, history: bool = True,
                    integrator: str = "semi_implicit_euler", picard_iterations: int = 8,
                    picard_tol: float = 1e-6, cic: int = 64, d: float = D_REF,
                    aspect: float = 4.0) -> Scene:
    rng = np.random.default_rng(seed)
    scale = (n / N_REF) ** (1.0 / 3.0)
    # column volume pi R^2 H with H = aspect * R, equal to the aspect-4 column's
    R = 0.1 * scale * (4.0 / aspect) ** (1.0 / 3.0)
    H = aspect * R
    box = (1.0 * scale, 1.0 * scale, max(0.5 * scale, 1.25 * H))
    diam = _diameters(rng, n, d, diameters)
    d_max = float(diam.max())
    # smallest spacing (>= d_max) whose first n sites fit in the cylinder
    spacing = max((math.pi * R * R * H / n) ** (1.0 / 3.0), d_max * 1.001)
    while True:
        sites = _cylinder_sites(n, spacing, R - 0.5 * d_max, 0.5 * spacing + 0.5 * d_max)
        if sites is not None and sites[-1, 2] + 0.5 * d_max <= box[2]:
            break
        spacing *= 0.995
        if spacing < d_max:
            raise ValueError("column does not fit the box")
    jitter = rng.uniform(-0.05 * d, 0.05 * d, size=(n, 3))
    pos = sites + jitter
    state = np.zeros((n, 6), np.float32)
    state[:, :3] = pos.astype(np.float32)
    cfg = ConfigSpec()
    _apply_common(cfg, box, d_max, d, mu=mu, restitution=restitution, k_n=k_n, density=density,
                  dt=dt, history=history, integrator=integrator,
                  picard_iterations=picard_iterations, picard_tol=picard_tol, cic=cic)
    return Scene(cfg, state, (0.5 * diam).astype(np.float32),
                 f"column_collapse n={n} d={diameters} mu={mu} H/R={aspect:g} {integrator}")


def perturbed_members(base: Scene, members: int, sigma: float = 50e-6,
                      seed: int = 7) -> list[Scene]:
    """Ensemble members of one scene: every grain moved by isotropic N(0, sigma^2)
    per axis, member m drawing from its own seed (seed, m). The reference perturbs
    by uniform +-p r per axis at initialization (src/particle_dynamics.cu:190-202);
    this Gaussian form is the ensemble's own generator."""
    out = []
    for m in range(members):
        rng = np.random.default_rng([seed, m])
        st = base.state.copy()
        st[:, :3] = (st[:, :3].astype(np.float64) +
                     rng.normal(0.0, sigma, size=(base.n, 3))).astype(np.float32)
        out.append(Scene(base.spec.copy(), st, base.radius.copy(), f"{base.name} member={m}"))
    return out


def ensemble_set_a(members: int = 64, n: int = N_REF, sigma: float = 50e-6,
                   seed: int = 7) -> list[Scene]:
    """64 perturbed copies of the 32,768-grain column (2,097,152 grains in all)."""
    return perturbed_members(column_collapse(n, diameters="uniform", cic=64), members,
                             sigma, seed)


def ensemble_set_b(scenes: int = 256, seed: int = 99, n_min: int = 4096,
                   n_max: int = 131072) -> list[Scene]:
    """Heterogeneous design: per scene n log-uniform in [n_min, n_max], aspect ratio
    H/R uniform in [1, 6] and friction uniform in [0, 0.8] (about 9.4 M grains for
    the default 256 scenes)."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), scenes)).astype(np.int64)
    aspects = rng.uniform(1.0, 6.0, scenes)
    mus = rng.uniform(0.0, 0.8, scenes)
    return [column_collapse(int(ns[k]), diameters="uniform", mu=float(mus[k]),
                            aspect=float(aspects[k]), cic=32, seed=int(seed * 1000 + k))
            for k in range(scenes)]


def dense_box(n: int = 1 << 24, *, phi: float = 0.55, seed: int = 2024, mu: float = 0.5,
              restitution: float = 0.5, k_n: float = 1e5, density: float = 2500.0,
              dt: float = 1e-5, history: bool = True, cic: int = 64) -> Scene:
    rng = np.random.default_rng(seed)
    box = (2.0, 2.0, 1.0)
    vol = box[0] * box[1] * box[2]
    d = (6.0 * phi * vol / (math.pi * n)) ** (1.0 / 3.0)
    a = (2.0 * (math.pi / 6.0) * d ** 3 / phi) ** (1.0 / 3.0)   # BCC: 2 sites per a^3
    # shrink the cell until the lattice inside the walls holds n sites (the overall
    # volume fraction stays phi: the lattice just fills the box a little less)
    while True:
        nx, ny, nz = (int(math.floor((L - d) / a)) for L in box)
        if 2 * nx * ny * nz >= n:
            break
        a *= 0.998
    base = np.stack(np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij"),
                    axis=-1).reshape(-1, 3)[:, ::-1].astype(np.float64)   # (x, y, z), z-major
    corner = base * a
    centre = corner + 0.5 * a
    sites = np.empty((2 * base.shape[0], 3))
    sites[0::2] = corner
    sites[1::2] = centre
    sites = sites[:n]
    if sites.shape[0] < n:
        raise ValueError("box too small for the requested grains")
    lo = np.array([-0.5 * box[0], -0.5 * box[1], 0.0]) + 0.5 * d + 0.02 * a
    pos = lo + sites + rng.uniform(-0.02 * d, 0.02 * d, size=(n, 3))
    state = np.zeros((n, 6), np.float32)
    state[:, :3] = pos.astype(np.float32)
    state[:, 3:] = rng.normal(0.0, 0.5, size=(n, 3)).astype(np.float32)
    cfg = ConfigSpec()
    _apply_common(cfg, box, d, d, mu=mu, restitution=restitution, k_n=k_n, density=density,
                  dt=dt, history=history, integrator="semi_implicit_euler",
                  picard_iterations=8, picard_tol=1e-6, cic=cic)
    return Scene(cfg, state, np.full(n, 0.5 * d, np.float32), f"dense_box n={n} phi={phi}")


def scene_for(workload: str, n: int | None = None, seed: int | None = None) -> Scene:
    """Named workloads used by bench.py and the tests."""
    kw = {} if seed is None else {"seed": seed}
    if workload == "collapse_32k":
        return column_collapse(n or N_REF, diameters="uniform", cic=64, **kw)
    if workload == "collapse_1m_sie_mu05":
        return column_collapse(n or (1 << 20), diameters="lognormal", mu=0.5, cic=128, **kw)
    if workload == "collapse_1m_sie_mu0":
        return column_collapse(n or (1 << 20), diameters="lognormal", mu=0.0, cic=128, **kw)
    if workload == "collapse_1m_picard_mu05":
        return column_collapse(n or (1 << 20), diameters="lognormal", mu=0.5, cic=128,
                               integrator="backward_euler_picard", **kw)
    if workload == "dense_16m":
        return dense_box(n or (1 << 24), **kw)
    raise ValueError(f"unknown workload '{workload}'")


BATCHED_WORKLOADS = ("ensemble_64x32k", "design_256")


def ensemble_for(workload: str) -> list[Scene]:
    """Named batched workloads: ensemble_64x32k (64 perturbed 32,768-grain columns)
    and design_256 (256 heterogeneous columns)."""
    if workload == "ensemble_64x32k":
        return ensemble_set_a()
    if workload == "design_256":
        return ensemble_set_b()
    raise ValueError(f"unknown batched workload '{workload}'")
