"""The reverse pass at the differentiable window's full size.

The 32,768-grain column (uniform diameters, mu = 0.5 with tangential springs, e = 0.5,
k_n = 1e5 N/m) after 12,000 steps: the lower column has reached the floor and is
collapsing, tens of thousands of springs are live (after 2,000 steps the lattice is still
falling without a single contact, so a window there would test free flight only). Then a
200-step window with checkpoints every 20 steps; loss = mean((rho_T - rho_target)^2) over
the 64^3 CIC mass field, the target from the same window with mu = 0.4, e = 0.6.

Two FP64 checks (tests/adjoint_torch.py, a torch float64 restatement of the step):
  * along the library's own FP32 trajectory: every step's vector-Jacobian product
    evaluated in FP64 at the library's recorded state and springs of that step, chained
    back from the loss. The library's FP32 gradients in e, k_n and v0 (every grain) must
    agree within 1e-3 relative: each parameter, v0 in three random directions and as a
    whole vector (relative L2 norm). dL/dmu within 1e-2: mu acts only through contacts
    that slide, and a sliding contact sits on the Coulomb cap by construction, so its
    stick/slip branch is a tie that FP32 and FP64 break differently (the two caps of one
    contact differ by up to 5e-4 relative where a shallow overlap loses digits in
    |delta| - r_i - r_j), and the two branches have different Jacobians;
  * along the FP64 trajectory of the same window: torch.autograd through the frozen
    FP64 window against its central finite differences (h = 1e-4, relative for k_n),
    within 1e-3. This pins the restatement itself.
The library's gradients are also printed against the FP64 trajectory's: 200 steps of a
collapsing column amplify the rounding difference of the two trajectories (a few percent
in dL/dmu on a B200), which is why the 1e-3 bar is taken along the library's own states.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import adjoint_torch as AT
from world_b200 import ParticleDynamics
from world_b200.adjoint import deposit, window
from world_b200.scenes import column_collapse

pytestmark = pytest.mark.gpu

RTOL = 1e-3


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_c4_window_gradients_match_fp64_adjoint_and_finite_differences():
    sc = column_collapse(32768, diameters="uniform", cic=64)
    cfg = sc.cfg
    cfg.kernel_timing = False
    ph = cfg.physics
    mu, e, k = float(ph.friction), float(ph.restitution), float(ph.normal_stiffness)
    steps, every = 200, 20
    sim = ParticleDynamics(cfg, state=sc.state, radius=sc.radius)
    sim.advance(12000)
    start = sim.get_state().reshape(-1, 6).copy()
    springs = sim.get_history()
    assert int(springs[0].sum()) > 10000
    n = sim.n
    size = (cfg.density_grid_size_x, cfg.density_grid_size_y, cfg.density_grid_size_z)
    assert size == (64, 64, 64)
    lo = [cfg.domain.x_min, cfg.domain.y_min, cfg.domain.z_min]
    hi = [cfg.domain.x_max, cfg.domain.y_max, cfg.domain.z_max]

    # target field: the same window with mu = 0.4, e = 0.6
    sim.set_contact_params(0.4, 0.6, k)
    sim.set_state(start)
    sim.set_history(*springs)
    sim.advance(steps)
    sim.compute_density_grid()
    target = torch.tensor(sim.host_density_grid[:sim.density_grid_nodes()].astype(np.float64),
                          device="cuda").reshape(size)
    sim.set_contact_params(mu, e, k)

    # the library's own trajectory, step by step (the window below repeats it exactly)
    model = AT.model_from_config(cfg, sc.radius, sim.grain_mass.copy())
    sim.set_state(start)
    sim.set_history(*springs)
    traj, sprs = [], []
    for t in range(steps + 1):
        traj.append(torch.tensor(sim.get_state().reshape(-1, 6), dtype=torch.float64,
                                 device="cuda"))
        sprs.append(AT.springs_from_rows(n, *sim.get_history()))
        if t < steps:
            sim.take_step()

    # the library: FP32 forward window with checkpoints, hand-written reverse pass
    sim.set_state(start)
    sim.set_history(*springs)
    xs = torch.tensor(start[:, :3], device="cuda")
    tv0 = torch.tensor(start[:, 3:], device="cuda", requires_grad=True)
    theta = torch.tensor([mu, e, k], dtype=torch.float64, requires_grad=True)
    x, v = window(sim, xs, tv0, theta, steps, every)
    grid = deposit(sim, x, v)
    loss32 = ((grid[0].double() - target) ** 2).mean()
    loss32.backward()
    g32_v0 = tv0.grad.double()
    g32_th = theta.grad.numpy().copy()
    sim.close()

    # FP64 adjoint along the library's trajectory
    m64 = model.mass
    th0 = torch.tensor([mu, e, k], dtype=torch.float64, device="cuda")
    ga_v0, _, ga_th = AT.adjoint_along(
        model, traj, sprs, th0,
        lambda x, v: ((AT.cic(x, v, m64, lo, hi, size)[0] - target) ** 2).mean())
    ga_th = ga_th.cpu().numpy()
    rel_th = [_rel(g32_th[a], ga_th[a]) for a in range(3)]
    for a in range(3):
        print(f"theta[{a}] along the library's states: library {g32_th[a]:.6e}  "
              f"fp64 {ga_th[a]:.6e}  rel {rel_th[a]:.2e}")
    whole_along = float((g32_v0 - ga_v0).norm() / ga_v0.norm())
    print(f"v0 gradient along the library's states, relative L2 difference: {whole_along:.3e}")
    rng_a = np.random.default_rng(9)
    rel_dirs = []
    for _ in range(3):
        dv = torch.tensor(rng_a.normal(size=(n, 3)), device="cuda")
        rel_dirs.append(_rel(float((g32_v0 * dv).sum()), float((ga_v0 * dv).sum())))
    print(f"v0 directions along the library's states: {rel_dirs}")
    assert rel_th[0] < 10 * RTOL
    assert rel_th[1] < RTOL and rel_th[2] < RTOL
    assert whole_along < RTOL
    assert max(rel_dirs) < RTOL

    # FP64: the same window on its own trajectory, recorded, then frozen
    x0 = torch.tensor(start[:, :3], dtype=torch.float64, device="cuda")
    v0 = torch.tensor(start[:, 3:], dtype=torch.float64, device="cuda")
    sp0 = AT.springs_from_rows(n, *springs)

    with torch.no_grad():
        _, _, pat = AT.run(model, x0, v0, sp0, th0[0], th0[1], th0[2], steps)
    assert sum(int(p["pairs"][0].numel()) for p in pat) > 100000

    def loss64(v_, th_):
        xT, vT, _ = AT.run(model, x0, v_, sp0, th_[0], th_[1], th_[2], steps, pattern=pat)
        return ((AT.cic(xT, vT, m64, lo, hi, size)[0] - target) ** 2).mean()

    tv = v0.clone().requires_grad_(True)
    tth = th0.clone().requires_grad_(True)
    l64 = loss64(tv, tth)
    l64.backward()
    g64_v0 = tv.grad
    g64_th = tth.grad.cpu().numpy()
    assert _rel(float(loss32), float(l64)) < 1e-2

    rng = np.random.default_rng(4)
    h = 1e-4
    with torch.no_grad():
        # parameters: FD (h relative for k_n), the FP64 adjoint, the library
        for a, step in ((0, h), (1, h), (2, h * k)):
            d = torch.zeros(3, dtype=torch.float64, device="cuda")
            d[a] = step
            fd = float((loss64(v0, th0 + d) - loss64(v0, th0 - d)) / (2 * step))
            print(f"theta[{a}] on the FP64 trajectory: library {g32_th[a]:.6e}  "
                  f"fp64 adjoint {g64_th[a]:.6e}  fd {fd:.6e}")
            assert _rel(g64_th[a], fd) < RTOL
        # v0 in random directions
        for _ in range(3):
            dv = torch.tensor(rng.normal(size=(n, 3)), device="cuda")
            fd = float((loss64(v0 + h * dv, th0) - loss64(v0 - h * dv, th0)) / (2 * h))
            a32 = float((g32_v0 * dv).sum())
            a64 = float((g64_v0 * dv).sum())
            print(f"v0 direction on the FP64 trajectory: library {a32:.6e}  "
                  f"fp64 adjoint {a64:.6e}  fd {fd:.6e}")
            assert _rel(a64, fd) < RTOL
    whole = float((g32_v0 - g64_v0).norm() / g64_v0.norm())
    print(f"v0 gradient, relative L2 difference library vs the FP64 trajectory: {whole:.3e}")
