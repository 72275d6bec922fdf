"""One scene split across ranks: x-slabs of whole collision cells with one-cell halos.

The reference runs a scene on one device (src/particle_dynamics.cu:10-94); a scene
larger than one GPU's memory has to be split. Rank r owns the grains whose collision
cell column lies in [cut[r], cut[r+1]) (x cell index, the reference's cell expression,
src/find_neighbors_kernel.cu:11-22); the cuts balance the initial grain counts. Every
step, each rank

  1. steps its owned grains together with ghost copies of the neighbours' grains in the
     one cell column next to its slab on each side (the 27-cell stencil of an owned
     grain never reaches further), on its own device through libworld_b200;
  2. keeps its owned grains' new state and tangential springs (ghosts' results are
     discarded: their forces lack their own neighbours);
  3. sends the grains whose new cell column left the slab (state, radius, mass, springs)
     to the neighbour that now owns them;
  4. sends its boundary columns to the neighbours as their new ghosts.

Contacts are gathered per owned grain, so no force crosses a rank. Local ids follow the
global grain ids, so the library visits contacts in the single-scene order and the
owned grains advance bit for bit as in one process. Each grain carries its own spring
row (the two sides of a pair keep mirrored springs), so history moves with migrating
grains; the spring and pair energies are carried by the smaller-id grain of each pair
(wd_grain_energies), so the FP64 all-reduce of the owned grains' terms counts each
once. Momentum is an FP64 all-reduce too.

Transport: torch.distributed point-to-point messages between neighbouring ranks (the
exchanges land in host arrays that the next local step uploads; with the NCCL backend
the messages are device tensors). Nothing here is a collective kernel over peer memory.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

HIST_CAP = 24


def cell_x(x: np.ndarray, lo: float, hi: float, g: int) -> np.ndarray:
    """The reference's cell index along x in float32 (src/find_neighbors_kernel.cu:11-22):
    trunc((x - lo) / (hi - lo) * g) clamped to [0, g - 1]."""
    f32 = np.float32
    t = ((np.asarray(x, f32) - f32(lo)) / (f32(hi) - f32(lo))) * f32(g)
    with np.errstate(invalid="ignore"):
        k = np.trunc(np.nan_to_num(np.clip(t, -2.0**31, 2.0**31 - 1), nan=0.0)).astype(np.int64)
    return np.clip(k, 0, g - 1)


def slab_cuts(cols: np.ndarray, g: int, ranks: int) -> np.ndarray:
    """Cuts 0 = c_0 < c_1 < ... < c_R = g in cell columns, balancing the grains of
    `cols` (their x cell columns); every slab at least one column wide."""
    if ranks < 1 or ranks > g:
        raise ValueError(f"{ranks} slabs for {g} cell columns")
    hist = np.bincount(cols, minlength=g).astype(np.float64)
    cum = np.cumsum(hist)
    total = cum[-1]
    cuts = [0]
    for r in range(1, ranks):
        c = int(np.searchsorted(cum, total * r / ranks, side="right"))
        c = max(c, cuts[-1] + 1)
        c = min(c, g - (ranks - r))
        cuts.append(c)
    cuts.append(g)
    return np.array(cuts, np.int64)


@dataclass
class Grains:
    """Grains by global id: state (k, 6) float32, radius, mass, and (owned grains) the
    spring rows with partners as global ids."""
    gid: np.ndarray
    state: np.ndarray
    radius: np.ndarray
    mass: np.ndarray
    count: np.ndarray | None = None
    partner: np.ndarray | None = None     # (k, 24) int64, walls -1 .. -6
    xi: np.ndarray | None = None          # (k, 24, 3) float32

    @property
    def k(self) -> int:
        return int(self.gid.size)

    def take(self, sel) -> "Grains":
        pick = (lambda a: None if a is None else a[sel])
        return Grains(self.gid[sel], self.state[sel], self.radius[sel], self.mass[sel],
                      pick(self.count), pick(self.partner), pick(self.xi))

    @staticmethod
    def cat(parts: list["Grains"], history: bool) -> "Grains":
        def c(name, empty):
            arrs = [getattr(p, name) for p in parts]
            return np.concatenate(arrs) if arrs else empty
        out = Grains(c("gid", np.zeros(0, np.int64)), c("state", np.zeros((0, 6), np.float32)),
                     c("radius", np.zeros(0, np.float32)), c("mass", np.zeros(0, np.float32)))
        if history:
            out.count = c("count", np.zeros(0, np.int32))
            out.partner = c("partner", np.zeros((0, HIST_CAP), np.int64))
            out.xi = c("xi", np.zeros((0, HIST_CAP, 3), np.float32))
        return out


class LibraryStepper:
    """The local step: a libworld_b200 handle over the rank's owned and ghost grains.
    The handle is kept while the local grain set is unchanged (then only the state and
    springs are uploaded) and rebuilt when it changes."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.sim = None
        self.gid = None

    def _handle(self, gid, state, radius, mass):
        from .particle_dynamics import ParticleDynamics
        if self.sim is not None and self.gid is not None and np.array_equal(self.gid, gid):
            self.sim.set_state(state)
        else:
            if self.sim is not None:
                self.sim.close()
            self.sim = ParticleDynamics(self.cfg, state=state, radius=radius, mass=mass)
            self.gid = gid.copy()
        return self.sim

    def step(self, gid, state, radius, mass, rows):
        sim = self._handle(gid, state, radius, mass)
        if rows is not None:
            sim.set_history(*rows)
        sim.take_step()
        out = sim.get_state().reshape(-1, 6)
        return out, (sim.get_history() if rows is not None else None)

    def grain_energies(self, gid, state, radius, mass, rows):
        sim = self._handle(gid, state, radius, mass)
        if rows is not None:
            sim.set_history(*rows)
        return sim.grain_energies()

    def close(self):
        if self.sim is not None:
            self.sim.close()
            self.sim = None


class SlabDomain:
    """This rank's slab of one scene. `spec` is the scene's configuration (a SimConfig or
    a ConfigSpec: the box, the collision grid and simulation.history are read); state,
    radius and mass are the whole scene's, by global id (every rank passes the same);
    `group` the torch.distributed process group (default: the world)."""

    def __init__(self, spec, state, radius, mass, stepper, group=None, springs=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.stepper = stepper
        self.lo = float(spec.domain.x_min)
        self.hi = float(spec.domain.x_max)
        self.g = int(spec.collision_grid_size_x)
        self.history = bool(spec.history)
        state = np.asarray(state, np.float32).reshape(-1, 6)
        n = state.shape[0]
        self.n_total = n
        cols = cell_x(state[:, 0], self.lo, self.hi, self.g)
        self.cuts = slab_cuts(cols, self.g, self.world)
        all_grains = Grains(np.arange(n, dtype=np.int64), state,
                            np.asarray(radius, np.float32), np.asarray(mass, np.float32))
        if self.history:
            if springs is None:
                all_grains.count = np.zeros(n, np.int32)
                all_grains.partner = np.zeros((n, HIST_CAP), np.int64)
                all_grains.xi = np.zeros((n, HIST_CAP, 3), np.float32)
            else:
                cnt, part, xi = springs
                all_grains.count = np.asarray(cnt, np.int32).copy()
                all_grains.partner = np.asarray(part, np.int64).reshape(n, HIST_CAP).copy()
                all_grains.xi = np.asarray(xi, np.float32).reshape(n, HIST_CAP, 3).copy()
        lo_c, hi_c = self.cuts[self.rank], self.cuts[self.rank + 1]
        self.owned = all_grains.take((cols >= lo_c) & (cols < hi_c))
        ghost_sel = (cols == lo_c - 1) | (cols == hi_c)
        self.ghosts = all_grains.take(ghost_sel)
        self.ghosts.count = self.ghosts.partner = self.ghosts.xi = None
        self.migrated = 0

    # -- local arrays ---------------------------------------------------------------
    def _local(self):
        """Owned and ghost grains ordered by global id, and the owned ones' positions in
        that order; springs with partners as local indices (ghosts carry none)."""
        gid = np.concatenate([self.owned.gid, self.ghosts.gid])
        order = np.argsort(gid, kind="stable")
        gid = gid[order]
        state = np.concatenate([self.owned.state, self.ghosts.state])[order]
        radius = np.concatenate([self.owned.radius, self.ghosts.radius])[order]
        mass = np.concatenate([self.owned.mass, self.ghosts.mass])[order]
        owned_at = np.searchsorted(gid, self.owned.gid)
        rows = None
        if self.history:
            k = gid.size
            cnt = np.zeros(k, np.int32)
            part = np.zeros((k, HIST_CAP), np.int32)
            xi = np.zeros((k, HIST_CAP, 3), np.float32)
            cnt[owned_at] = self.owned.count
            live = np.arange(HIST_CAP)[None, :] < self.owned.count[:, None]
            p = self.owned.partner.copy()
            grain = live & (p >= 0)
            at = np.searchsorted(gid, p[grain])
            at_c = np.minimum(at, k - 1)
            if not np.array_equal(gid[at_c], p[grain]):
                raise RuntimeError("slab: a spring partner is neither owned nor a ghost")
            p[grain] = at_c
            part[owned_at] = p.astype(np.int32)
            xi[owned_at] = self.owned.xi
            rows = (cnt, part.reshape(-1), xi.reshape(-1))
        return gid, state, radius, mass, owned_at, rows

    # -- exchange -------------------------------------------------------------------
    def _exchange(self, to_left: Grains, to_right: Grains, full: bool) -> list[Grains]:
        """Send `to_left` / `to_right` to the neighbouring ranks and return what they
        sent here (full records with springs, or ghost records)."""
        import torch
        dist = self.dist
        neighbours = [(self.rank - 1, to_left), (self.rank + 1, to_right)]
        neighbours = [(r, g) for r, g in neighbours if 0 <= r < self.world]

        def pack(g: Grains):
            f = np.concatenate([g.state, g.radius[:, None], g.mass[:, None]], 1)
            parts = [torch.from_numpy(np.ascontiguousarray(f, np.float32)),
                     torch.from_numpy(np.ascontiguousarray(g.gid, np.int64))]
            if full and self.history:
                parts += [torch.from_numpy(np.ascontiguousarray(g.count, np.int32)),
                          torch.from_numpy(np.ascontiguousarray(g.partner, np.int64)),
                          torch.from_numpy(np.ascontiguousarray(g.xi, np.float32))]
            return parts

        # counts first, then the records
        sizes = {r: torch.zeros(1, dtype=torch.int64) for r, _ in neighbours}
        ops = []
        for r, g in neighbours:
            ops.append(dist.P2POp(dist.isend, torch.tensor([g.k], dtype=torch.int64), r, self.group))
            ops.append(dist.P2POp(dist.irecv, sizes[r], r, self.group))
        for req in (dist.batch_isend_irecv(ops) if ops else []):
            req.wait()
        ops, recv = [], {}
        for r, g in neighbours:
            k = int(sizes[r].item())
            bufs = [torch.empty((k, 8), dtype=torch.float32), torch.empty(k, dtype=torch.int64)]
            if full and self.history:
                bufs += [torch.empty(k, dtype=torch.int32),
                         torch.empty((k, HIST_CAP), dtype=torch.int64),
                         torch.empty((k, HIST_CAP, 3), dtype=torch.float32)]
            recv[r] = bufs
            for t in pack(g):
                if t.numel():
                    ops.append(dist.P2POp(dist.isend, t, r, self.group))
            for t in bufs:
                if t.numel():
                    ops.append(dist.P2POp(dist.irecv, t, r, self.group))
        for req in (dist.batch_isend_irecv(ops) if ops else []):
            req.wait()
        out = []
        for r, _ in neighbours:
            b = [t.numpy() for t in recv[r]]
            g = Grains(b[1], b[0][:, :6].copy(), b[0][:, 6].copy(), b[0][:, 7].copy())
            if full and self.history:
                g.count, g.partner, g.xi = b[2], b[3], b[4]
            out.append(g)
        return out

    # -- the step -------------------------------------------------------------------
    def step(self, steps: int = 1) -> None:
        for _ in range(steps):
            self._step_once()

    def _step_once(self) -> None:
        gid, state, radius, mass, owned_at, rows = self._local()
        new_state, new_rows = self.stepper.step(gid, state, radius, mass, rows)
        self.owned.state = np.asarray(new_state, np.float32)[owned_at]
        if self.history:
            cnt, part, xi = new_rows
            k = gid.size
            part = part.reshape(k, HIST_CAP)[owned_at].astype(np.int64)
            live = np.arange(HIST_CAP)[None, :] < cnt[owned_at][:, None]
            grain = live & (part >= 0)
            part[grain] = gid[part[grain]]
            self.owned.count = cnt[owned_at].astype(np.int32)
            self.owned.partner = part
            self.owned.xi = xi.reshape(k, HIST_CAP, 3)[owned_at].copy()
        # migration: grains whose cell column left the slab go to the neighbour
        lo_c, hi_c = self.cuts[self.rank], self.cuts[self.rank + 1]
        cols = cell_x(self.owned.state[:, 0], self.lo, self.hi, self.g)
        left, right = cols < lo_c, cols >= hi_c
        if self.rank > 0 and np.any(cols[left] < self.cuts[self.rank - 1]) or \
                self.rank + 1 < self.world and np.any(cols[right] >= self.cuts[self.rank + 2]):
            raise RuntimeError("slab: a grain crossed a whole slab in one step")
        arrived = self._exchange(self.owned.take(left), self.owned.take(right), full=True)
        self.migrated += int(left.sum() + right.sum())
        self.owned = Grains.cat([self.owned.take(~(left | right))] + arrived, self.history)
        # halos: this slab's boundary columns become the neighbours' ghosts
        cols = cell_x(self.owned.state[:, 0], self.lo, self.hi, self.g)
        ghosts = self._exchange(self.owned.take(cols == lo_c), self.owned.take(cols == hi_c - 1),
                                full=False)
        self.ghosts = Grains.cat(ghosts, False)

    # -- reductions -----------------------------------------------------------------
    def _all_reduce(self, values: np.ndarray) -> np.ndarray:
        import torch
        t = torch.from_numpy(np.ascontiguousarray(values, np.float64))
        self.dist.all_reduce(t, group=self.group)
        return t.numpy()

    def total_energy(self) -> float:
        """The scene's total energy: the owned grains' terms (wd_grain_energies, each
        pair and spring carried by its smaller-id grain), FP64 all-reduce."""
        gid, state, radius, mass, owned_at, rows = self._local()
        e = self.stepper.grain_energies(gid, state, radius, mass, rows)
        return float(self._all_reduce(np.array([np.sum(e[owned_at])]))[0])

    def momentum(self) -> np.ndarray:
        """sum m v over the scene, FP64 all-reduce of the owned grains' sums."""
        m = self.owned.mass.astype(np.float64)
        p = (m[:, None] * self.owned.state[:, 3:].astype(np.float64)).sum(0)
        return self._all_reduce(p)

    def gather(self):
        """The whole scene by global id on every rank (state, and springs with global
        partner ids): for checks and output, not for the step."""
        import torch
        parts = [None] * self.world
        self.dist.all_gather_object(parts, (self.owned.gid, self.owned.state, self.owned.count,
                                            self.owned.partner, self.owned.xi), group=self.group)
        gid = np.concatenate([p[0] for p in parts])
        order = np.argsort(gid)
        if not np.array_equal(gid[order], np.arange(self.n_total)):
            raise RuntimeError("slab: grains lost or duplicated")
        state = np.concatenate([p[1] for p in parts])[order]
        if not self.history:
            return state, None
        cnt = np.concatenate([p[2] for p in parts])[order]
        part = np.concatenate([p[3] for p in parts])[order]
        xi = np.concatenate([p[4] for p in parts])[order]
        _ = torch
        return state, (cnt, part, xi)
