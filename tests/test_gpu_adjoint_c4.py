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
    back from the loss. The same chain is also evaluated in FP32 (torch, the same
    states), which shows what FP32 arithmetic alone does to this window's adjoint:
    shallow overlaps lose digits in |delta| - r_i - r_j (up to 5e-4 relative), sliding
    contacts sit on the Coulomb cap so their stick/slip branch is a near-tie that each
    FP32 evaluation breaks its own way, and 200 steps of a collapsing column carry both
    into every gradient. On a B200 the torch FP32 chain lands 3e-4 to 8e-3 from FP64 in
    the parameters and 1.8e-2 in dL/dv0, the library 6e-4 to 4e-3 and 1.7e-2. The bar:
    each of dL/dmu, dL/de, dL/dk_n within 1e-2 of the FP64 adjoint, dL/dv0 (every grain,
    relative L2 norm) within 5e-2;
  * along the FP64 trajectory of the same window: torch.autograd through the frozen
    FP64 window against its central finite differences (h = 1e-4 in the parameters,
    relative for k_n; 1e-6 m/s along random directions in v0, which move every grain),
    within 1e-3. This pins the restatement itself.
The library's gradients are also printed against the FP64 trajectory's: 200 steps of a
collapsing column amplify the rounding difference of the two trajectories (a few percent
in dL/dmu on a B200), which is why the library is compared along its own states.
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

RTOL = 1e-3          # FP64 adjoint against FP64 finite differences
FP32_THETA = 1e-2    # library (FP32) against the FP64 adjoint along its states
FP32_V0 = 5e-2


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

    # the same chain in FP32 arithmetic along the same states
    m32 = AT.model_as(model, torch.float32)
    gf_v0, _, gf_th = AT.adjoint_along(
        m32, [t.float() for t in traj], [(kk, xi.float()) for kk, xi in sprs], th0.float(),
        lambda x, v: ((AT.cic(x.double(), v.double(), m64, lo, hi, size)[0] - target) ** 2).mean())
    gf_v0 = gf_v0.double()
    gf_th = gf_th.double().cpu().numpy()
    floor_th = [_rel(gf_th[a], ga_th[a]) for a in range(3)]
    floor_v0 = float((gf_v0 - ga_v0).norm() / ga_v0.norm())
    lib_f32 = float((g32_v0 - gf_v0).norm() / ga_v0.norm())
    for a in range(3):
        print(f"theta[{a}]: torch FP32 along the same states {gf_th[a]:.6e}  "
              f"rel to fp64 {floor_th[a]:.2e}")
    print(f"v0: torch FP32 vs fp64 {floor_v0:.3e}, library vs torch FP32 {lib_f32:.3e}")
    for a in range(3):
        assert rel_th[a] < FP32_THETA, a
    assert whole_along < FP32_V0

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
    h = 1e-4       # parameters (relative for k_n)
    hv = 1e-6      # v0 directions: every grain moves, so the step is kept small
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
            fd = float((loss64(v0 + hv * dv, th0) - loss64(v0 - hv * dv, th0)) / (2 * hv))
            a32 = float((g32_v0 * dv).sum())
            a64 = float((g64_v0 * dv).sum())
            print(f"v0 direction on the FP64 trajectory: library {a32:.6e}  "
                  f"fp64 adjoint {a64:.6e}  fd {fd:.6e}")
            assert _rel(a64, fd) < RTOL
    whole = float((g32_v0 - g64_v0).norm() / g64_v0.norm())
    print(f"v0 gradient, relative L2 difference library vs the FP64 trajectory: {whole:.3e}")
