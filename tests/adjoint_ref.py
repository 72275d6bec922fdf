"""FP64 restatement of the semi-implicit Euler DEM step, for checking the reverse pass.

Vectorised numpy over brute-force pairs (small n only): gravity, the six walls, pair
contacts with the normal spring-dashpot, and either the reference's viscous friction or
the tangential spring with per-pair history (the library's extension), then
v' = v + dt F / m, x' = x + dt v'. The same laws as world_b200/csrc/wd_device.cuh and
oracle/dem_oracle.c, in double precision and in no particular summation order.

A run records its contact pattern: per step the wall and pair contacts and the branch
each took (clamp at max_force, Coulomb slip, viscous cap). Replaying with that pattern
frozen makes the step a smooth function of (x0, v0, mu, e, k_n), whose central finite
differences pin the library's adjoint. Test infrastructure only.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Model:
    radius: np.ndarray
    mass: np.ndarray
    dt: float
    gravity: float
    wall_lo: np.ndarray
    wall_hi: np.ndarray
    max_force: float          # inf: no clamp
    history: bool
    kt_fixed: float = 0.0     # > 0: physics.tangential_stiffness; else 2/7 k_n


@dataclass
class StepPattern:
    walls: list = field(default_factory=list)   # (a, up, idx, clamp, branch)
    pairs: tuple | None = None                  # (I, J, clamp, branch)


def damping(e: float, k, m):
    if e <= 0.0:
        return 2.0 * np.sqrt(k * m)
    if e >= 1.0:
        return 0.0 * m
    L = math.log(e)
    return -2.0 * np.sqrt(m * k) * L / math.sqrt(L * L + math.pi * math.pi)


def _friction(model, F, idx, vt, nrm, limit, c, partner, springs, new, branch, k, kt):
    """Adds the friction of contacts idx (rows of vt, nrm, limit, c) to F; returns the
    branch flags (slip for springs, capped / active for viscous)."""
    if model.history:
        xi = np.array([springs.get((int(i), int(p)), np.zeros(3)) for i, p in zip(idx, partner)])
        xi = xi.reshape(-1, 3)
        xn = (xi * nrm).sum(1, keepdims=True)
        xi = xi - xn * nrm + model.dt * vt
        ft = -kt * xi
        fmag = np.sqrt((ft * ft).sum(1))
        slip = fmag > limit if branch is None else branch
        s = np.where(slip, limit / np.where(fmag > 0, fmag, 1.0), 1.0)[:, None]
        ft = ft * s
        xi = xi * s
        np.add.at(F, idx, ft)
        for r, (i, p) in enumerate(zip(idx, partner)):
            new[(int(i), int(p))] = xi[r]
        return slip
    v = np.sqrt((vt * vt).sum(1))
    if branch is None:
        active = v >= 1e-8
        capped = limit < c * v
        branch = np.stack([active, capped], 1)
    active, capped = branch[:, 0], branch[:, 1]
    mag = np.where(capped, limit, c * v)
    vs = np.where(active, v, 1.0)
    np.add.at(F, idx, -np.where(active, mag / vs, 0.0)[:, None] * vt)
    return branch


def step(model: Model, x, v, springs: dict, mu: float, e: float, k: float,
         pat: StepPattern | None = None):
    """One step; returns (x', v', springs', pattern)."""
    n = x.shape[0]
    r, m = model.radius, model.mass
    kt = model.kt_fixed if model.kt_fixed > 0 else (2.0 / 7.0) * k
    F = np.zeros((n, 3))
    F[:, 2] -= m * model.gravity
    new: dict = {}
    out = StepPattern()
    # walls
    wi = 0
    for a in range(3):
        for up in (0, 1):
            dl = (model.wall_hi[a] - x[:, a]) - r if up else (x[:, a] - model.wall_lo[a]) - r
            if pat is None:
                idx = np.nonzero(dl < 0)[0]
                raw = -k * dl[idx]
                clamp = raw > model.max_force
            else:
                _, _, idx, clamp, _ = pat.walls[wi]
                raw = -k * dl[idx]
            fl = np.where(clamp, model.max_force, raw)
            sign = -1.0 if up else 1.0
            np.add.at(F[:, a], idx, sign * fl)
            c = damping(e, k, m[idx])
            np.add.at(F[:, a], idx, -c * v[idx, a])
            vt = v[idx].copy()
            vt[:, a] = 0.0
            nrm = np.zeros((idx.size, 3))
            nrm[:, a] = sign
            partner = np.full(idx.size, (-2 - 2 * a) if up else (-1 - 2 * a))
            branch = _friction(model, F, idx, vt, nrm, mu * fl, c, partner, springs, new,
                               None if pat is None else pat.walls[wi][4], k, kt)
            out.walls.append((a, up, idx, clamp, branch))
            wi += 1
    # pairs (ordered: the force on I from J)
    if pat is None:
        d_all = x[:, None, :] - x[None, :, :]
        dist_all = np.sqrt((d_all ** 2).sum(-1)) - r[:, None] - r[None, :]
        np.fill_diagonal(dist_all, 1.0)
        I, J = np.nonzero(dist_all < 0)
    else:
        I, J = pat.pairs[0], pat.pairs[1]
    d = x[I] - x[J]
    norm = np.sqrt((d * d).sum(1))
    nrm = d / norm[:, None]
    dist = norm - r[I] - r[J]
    raw = -k * dist
    clamp = raw > model.max_force if pat is None else pat.pairs[2]
    fp = np.where(clamp, model.max_force, raw)
    np.add.at(F, I, fp[:, None] * nrm)
    mred = m[I] * m[J] / (m[I] + m[J])
    c = damping(e, k, mred)
    vr = v[I] - v[J]
    vn = (vr * nrm).sum(1)
    np.add.at(F, I, -(c * vn)[:, None] * nrm)
    vt = vr - vn[:, None] * nrm
    branch = _friction(model, F, I, vt, nrm, mu * fp, c, J, springs, new,
                       None if pat is None else pat.pairs[3], k, kt)
    out.pairs = (I, J, clamp, branch)
    v1 = v + model.dt * F / m[:, None]
    x1 = x + model.dt * v1
    return x1, v1, new, out


def run(model: Model, x0, v0, mu, e, k, steps: int, pattern: list | None = None):
    """(x_T, v_T, pattern) after `steps` steps; with a pattern the branches are frozen."""
    x, v, springs = np.array(x0, np.float64), np.array(v0, np.float64), {}
    rec = []
    for t in range(steps):
        x, v, springs, p = step(model, x, v, springs, mu, e, k, None if pattern is None else pattern[t])
        rec.append(p)
    return x, v, rec


def cic(x, v, mass, lo, hi, size):
    """Node-centred CIC of mass and momentum (4, nx, ny, nz) in FP64, the weights of
    src/density_grid_kernel.cu:25-83."""
    g = np.zeros((4, *size))
    h = [(hi[a] - lo[a]) / (size[a] - 1) for a in range(3)]
    for p in range(x.shape[0]):
        if mass[p] == 0:
            continue
        idx, w = [], []
        for a in range(3):
            u = (x[p, a] - lo[a]) / h[a]
            b = math.floor(u)
            f = u - b
            idx.append((min(size[a] - 1, max(0, b)), min(size[a] - 1, max(0, b + 1))))
            w.append((1.0 - f, f))
        for cx in range(2):
            for cy in range(2):
                for cz in range(2):
                    ww = w[0][cx] * w[1][cy] * w[2][cz]
                    node = (idx[0][cx], idx[1][cy], idx[2][cz])
                    g[0][node] += mass[p] * ww
                    for a in range(3):
                        g[1 + a][node] += mass[p] * v[p, a] * ww
    return g
