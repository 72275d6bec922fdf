"""FP64 restatement of the semi-implicit Euler DEM step in torch, for checking the reverse
pass at the differentiable window's full size (32,768 grains, 200 steps).

The laws are those of tests/adjoint_ref.py (and world_b200/csrc/wd_device.cuh): gravity,
the six walls and pair contacts with the normal spring, the dashpot and the tangential
spring with per-pair history (Coulomb cap with rescale on slip), then v' = v + dt F / m,
x' = x + dt v'. Here they run vectorised on the device in float64: candidate pairs come
from a cell grid whose cell is at least the largest contact distance, and each contact's
spring is carried from the step before through its (grain, partner) key.

A recorded run keeps, per step, its contacts and the branch each took (clamp at
max_force, Coulomb slip); replaying with that pattern frozen makes the window a smooth
function of (x0, v0, mu, e, k_n). Central finite differences of the replay, and
torch.autograd through it (the FP64 adjoint), both pin the library's FP32 adjoint.
Test infrastructure only.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

PI = math.pi


@dataclass
class TorchModel:
    radius: torch.Tensor      # (n,) float64
    mass: torch.Tensor        # (n,) float64
    dt: float
    gravity: float
    wall_lo: tuple
    wall_hi: tuple
    max_force: float          # inf: no clamp
    kt_fixed: float = 0.0     # > 0: physics.tangential_stiffness; else 2/7 k_n

    @property
    def n(self) -> int:
        return int(self.radius.numel())


def model_from_config(cfg, radius, mass, device="cuda") -> TorchModel:
    ph = cfg.physics
    return TorchModel(
        radius=torch.as_tensor(radius, dtype=torch.float64, device=device),
        mass=torch.as_tensor(mass, dtype=torch.float64, device=device),
        dt=float(cfg.dt), gravity=float(ph.gravity),
        wall_lo=(float(ph.wall_x_min), float(ph.wall_y_min), float(ph.floor_z)),
        wall_hi=(float(ph.wall_x_max), float(ph.wall_y_max), float(ph.ceiling_z)),
        max_force=float(ph.max_force) if ph.max_force > 0 else math.inf,
        kt_fixed=float(ph.tangential_stiffness))


def model_as(model: TorchModel, dtype) -> TorchModel:
    """The same model with radius and mass in `dtype`: with float32 states and springs,
    step() and adjoint_along() then evaluate every step in float32."""
    return TorchModel(radius=model.radius.to(dtype), mass=model.mass.to(dtype), dt=model.dt,
                      gravity=model.gravity, wall_lo=model.wall_lo, wall_hi=model.wall_hi,
                      max_force=model.max_force, kt_fixed=model.kt_fixed)


def damping(e, k, m):
    """reference src/compute_rhs_kernel.cu:41-47 for 0 < e < 1."""
    L = torch.log(e)
    return -2.0 * torch.sqrt(m * k) * L / torch.sqrt(L * L + PI * PI)


def _keys(n: int, grain: torch.Tensor, partner: torch.Tensor) -> torch.Tensor:
    """(grain, partner) as one int64; walls are partners -1 .. -6."""
    return grain.to(torch.int64) * (n + 8) + (partner.to(torch.int64) + 8)


def springs_from_rows(n, count, partner, xi, device="cuda"):
    """The library's spring rows (count[n], partner[n*24], xi[n*24*3], by grain id) as
    sorted keys and float64 springs."""
    cap = partner.size // n
    count_t = torch.as_tensor(count, device=device).to(torch.int64)
    live = torch.arange(cap, device=device)[None, :] < count_t[:, None]
    grain = torch.arange(n, device=device)[:, None].expand(n, cap)[live]
    part = torch.as_tensor(partner, device=device).reshape(n, cap)[live]
    x = torch.as_tensor(xi, device=device).reshape(n, cap, 3)[live].to(torch.float64)
    keys = _keys(n, grain, part)
    order = torch.argsort(keys)
    return keys[order], x[order]


def candidate_pairs(model: TorchModel, x: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """Ordered pairs (i, j), i != j, in the same or adjacent cells of a grid whose cell is
    at least the largest contact distance; every contact is among them."""
    n = model.n
    lo = x.min(0).values - 1e-9
    cs = 2.0 * float(model.radius.max()) * 1.01
    c = torch.floor((x - lo) / cs).to(torch.int64)
    g = c.max(0).values + 1
    key = (c[:, 0] * g[1] + c[:, 1]) * g[2] + c[:, 2]
    order = torch.argsort(key)
    ncell = int(g[0] * g[1] * g[2])
    counts = torch.bincount(key, minlength=ncell)
    start = torch.cumsum(counts, 0) - counts
    occ = int(counts.max())
    I_all, J_all = [], []
    ii = torch.arange(n, device=x.device)
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                nc = c + torch.tensor([dx, dy, dz], device=x.device)
                ok = ((nc >= 0) & (nc < g)).all(1)
                nk = torch.where(ok, (nc[:, 0] * g[1] + nc[:, 1]) * g[2] + nc[:, 2], 0)
                st, cn = start[nk], torch.where(ok, counts[nk], 0)
                for m in range(occ):
                    sel = m < cn
                    j = order[torch.clamp(st + m, max=n - 1)]
                    sel = sel & (j != ii)
                    I_all.append(ii[sel])
                    J_all.append(j[sel])
    return torch.cat(I_all), torch.cat(J_all)


def step(model: TorchModel, x, v, sp_keys, sp_xi, mu, e, k, pat=None):
    """One step. sp_keys (sorted) / sp_xi: the springs entering the step. Returns
    (x', v', keys', springs', pattern); with `pat` the contacts and branches are frozen."""
    n = model.n
    dev = x.device
    r, m = model.radius, model.mass
    kt = model.kt_fixed if model.kt_fixed > 0 else (2.0 / 7.0) * k
    F = torch.zeros_like(x)
    F[:, 2] = -m * model.gravity
    rec = {} if pat is None else pat
    # walls: lower a -> partner -1 - 2a, normal +e_a; upper -> -2 - 2a, normal -e_a
    g_list, p_list, n_list, f_list, c_list = [], [], [], [], []
    for a in range(3):
        for up in (0, 1):
            name = f"w{a}{up}"
            if pat is None:
                dl = (model.wall_hi[a] - x[:, a]) - r if up else (x[:, a] - model.wall_lo[a]) - r
                idx = torch.nonzero(dl < 0).flatten()
                clamp = (-k * dl[idx]) > model.max_force
                rec[name] = (idx, clamp)
            idx, clamp = rec[name]
            dl = (model.wall_hi[a] - x[idx, a]) - r[idx] if up else (x[idx, a] - model.wall_lo[a]) - r[idx]
            fl = torch.where(clamp, torch.full_like(dl, model.max_force), -k * dl)
            sign = -1.0 if up else 1.0
            cw = damping(e, k, m[idx])
            fa = sign * fl - cw * v[idx, a]
            F = F.index_add(0, idx, torch.nn.functional.one_hot(torch.full_like(idx, a), 3).to(x.dtype) * fa[:, None])
            nrm = torch.zeros((idx.numel(), 3), dtype=x.dtype, device=dev)
            nrm[:, a] = sign
            vt = v[idx] * (1.0 - torch.nn.functional.one_hot(torch.full_like(idx, a), 3).to(x.dtype))
            g_list.append(idx)
            p_list.append(torch.full_like(idx, (-2 - 2 * a) if up else (-1 - 2 * a)))
            n_list.append(nrm)
            f_list.append(fl)
            c_list.append(vt)
    # pairs (ordered: the force on I from J)
    if pat is None:
        I, J = candidate_pairs(model, x.detach())
        d = x[I] - x[J]
        dist = torch.sqrt((d * d).sum(1)) - r[I] - r[J]
        keep = dist < 0
        I, J = I[keep], J[keep]
        clamp = (-k * dist[keep]) > model.max_force
        rec["pairs"] = (I, J, clamp)
    I, J, clamp = rec["pairs"]
    d = x[I] - x[J]
    norm = torch.sqrt((d * d).sum(1))
    nrm = d / norm[:, None]
    dist = norm - r[I] - r[J]
    fp = torch.where(clamp, torch.full_like(dist, model.max_force), -k * dist)
    mred = m[I] * m[J] / (m[I] + m[J])
    c = damping(e, k, mred)
    vr = v[I] - v[J]
    vn = (vr * nrm).sum(1)
    F = F.index_add(0, I, (fp - c * vn)[:, None] * nrm)
    vt_p = vr - vn[:, None] * nrm
    # tangential springs of all contacts (walls, then pairs)
    grain = torch.cat(g_list + [I])
    partner = torch.cat(p_list + [J])
    nrm_all = torch.cat(n_list + [nrm])
    limit = mu * torch.cat(f_list + [fp])
    vt = torch.cat(c_list + [vt_p])
    keys = _keys(n, grain, partner)
    if pat is None:
        pos = torch.searchsorted(sp_keys, keys).clamp(max=max(sp_keys.numel() - 1, 0))
        found = (sp_keys.numel() > 0) & (sp_keys[pos] == keys) if sp_keys.numel() else \
            torch.zeros_like(keys, dtype=torch.bool)
        rec["prev"] = torch.where(found, pos, torch.full_like(pos, -1))
    prev = rec["prev"]
    xi0 = torch.where((prev >= 0)[:, None], sp_xi[prev.clamp(min=0)] if sp_xi.numel() else
                      torch.zeros_like(vt), torch.zeros_like(vt))
    xn = (xi0 * nrm_all).sum(1, keepdim=True)
    xi = xi0 - xn * nrm_all + model.dt * vt
    ft = -kt * xi
    fmag = torch.sqrt((ft * ft).sum(1))
    if pat is None:
        rec["slip"] = fmag > limit
    slip = rec["slip"]
    s = torch.where(slip, limit / torch.where(fmag > 0, fmag, torch.ones_like(fmag)),
                    torch.ones_like(fmag))[:, None]
    ft = ft * s
    xi = xi * s
    F = F.index_add(0, grain, ft)
    v1 = v + model.dt * F / m[:, None]
    x1 = x + model.dt * v1
    if pat is None:
        rec["order"] = torch.argsort(keys)
    order = rec["order"]
    return x1, v1, keys[order], xi[order], rec


def run(model: TorchModel, x0, v0, springs0, mu, e, k, steps: int, pattern=None):
    """(x_T, v_T, pattern) after `steps` steps from (x0, v0) and the initial springs
    (sorted keys, float64 springs); with a pattern the contacts and branches are frozen."""
    x, v = x0, v0
    keys, xi = springs0
    rec = []
    for t in range(steps):
        x, v, keys, xi, p = step(model, x, v, keys, xi, mu, e, k,
                                 None if pattern is None else pattern[t])
        rec.append(p)
    return x, v, rec


def cic(x, v, mass, lo, hi, size):
    """Node-centred CIC of mass and momentum, (4, nx, ny, nz) float64, the weights of
    src/density_grid_kernel.cu:25-83, differentiable in x and v."""
    dev = x.device
    nodes = size[0] * size[1] * size[2]
    h = [(hi[a] - lo[a]) / (size[a] - 1) for a in range(3)]
    idx, w = [], []
    for a in range(3):
        u = (x[:, a] - lo[a]) / h[a]
        b = torch.floor(u.detach())
        f = u - b
        bi = b.to(torch.int64)
        idx.append((bi.clamp(0, size[a] - 1), (bi + 1).clamp(0, size[a] - 1)))
        w.append((1.0 - f, f))
    out = torch.zeros((4, nodes), dtype=x.dtype, device=dev)
    live = mass != 0
    chan = torch.cat([mass[:, None], mass[:, None] * v], 1)       # (n, 4)
    for cx in range(2):
        for cy in range(2):
            for cz in range(2):
                ww = w[0][cx] * w[1][cy] * w[2][cz]
                node = (idx[0][cx] * size[1] + idx[1][cy]) * size[2] + idx[2][cz]
                contrib = torch.where(live[:, None], chan * ww[:, None], torch.zeros_like(chan))
                out = out.index_add(1, node, contrib.T)
    return out.reshape(4, *size)


def adjoint_along(model: TorchModel, traj, springs, theta, loss_of_end):
    """The FP64 adjoint of a window along a given trajectory: traj[t] (n, 6) is the state
    entering step t (t = 0 .. T, traj[T] the end), springs[t] the (sorted keys, springs)
    entering step t (t = 0 .. T - 1; more entries are ignored). Each step's
    vector-Jacobian product is evaluated at those states, with its own contact and
    stick/slip decisions there, and chained back from loss_of_end(x_T, v_T). Returns
    (dL/dv0, dL/dx0, dL/dtheta)."""
    steps = len(traj) - 1
    xT = traj[-1][:, :3].clone().requires_grad_(True)
    vT = traj[-1][:, 3:].clone().requires_grad_(True)
    loss_of_end(xT, vT).backward()
    gx = xT.grad if xT.grad is not None else torch.zeros_like(xT)
    gv = vT.grad if vT.grad is not None else torch.zeros_like(vT)
    g_keys, g_xi = None, None
    g_th = torch.zeros(3, dtype=theta.dtype, device=theta.device)
    for t in reversed(range(steps)):
        x = traj[t][:, :3].clone().requires_grad_(True)
        v = traj[t][:, 3:].clone().requires_grad_(True)
        keys_t, xi_t = springs[t]
        xi_t = xi_t.clone().requires_grad_(True)
        th = theta.clone().requires_grad_(True)
        x1, v1, keys1, xi1, _ = step(model, x, v, keys_t, xi_t, th[0], th[1], th[2])
        outs, grads = [x1, v1], [gx, gv]
        if g_xi is not None and xi1.numel() and g_keys.numel():
            at = torch.searchsorted(g_keys, keys1).clamp(max=g_keys.numel() - 1)
            hit = (g_keys[at] == keys1)[:, None]
            outs.append(xi1)
            grads.append(torch.where(hit, g_xi[at], torch.zeros_like(xi1)))
        torch.autograd.backward(outs, grads)
        gx = x.grad if x.grad is not None else torch.zeros_like(x)
        gv = v.grad if v.grad is not None else torch.zeros_like(v)
        g_keys = keys_t
        g_xi = xi_t.grad if xi_t.grad is not None else torch.zeros_like(xi_t)
        if th.grad is not None:
            g_th = g_th + th.grad
    return gv, gx, g_th


def record_trajectory(model: TorchModel, x0, v0, springs0, theta, steps: int):
    """The FP64 run's own states and springs entering each step (for adjoint_along)."""
    x, v = x0, v0
    keys, xi = springs0
    traj, sprs = [torch.cat([x, v], 1)], []
    with torch.no_grad():
        for _ in range(steps):
            sprs.append((keys, xi))
            x, v, keys, xi, _ = step(model, x, v, keys, xi, theta[0], theta[1], theta[2])
            traj.append(torch.cat([x, v], 1))
    sprs.append((keys, xi))
    return traj, sprs
