"""The reverse pass at the differentiable window's full size.

The 32,768-grain column (uniform diameters, mu = 0.5 with tangential springs, e = 0.5,
k_n = 1e5 N/m) after 12,000 steps: the lower column has reached the floor and is
collapsing, tens of thousands of springs are live (after 2,000 steps the lattice is still
falling without a single contact, so a window there would test free flight only). Then a
200-step window with checkpoints every 20 steps; loss = mean((rho_T - rho_target)^2) over
the 64^3 CIC mass field, the target from the same window with mu = 0.4, e = 0.6.

The library's FP32 gradients in (mu, e, k_n) and in v0 (every grain) are checked against
  * central finite differences (h = 1e-4, relative for k_n) of the FP64 restatement
    (tests/adjoint_torch.py) with its contact set and branches frozen, and
  * the FP64 adjoint: torch.autograd through that same frozen FP64 window,
within 1e-3 relative: the parameters each, v0 in three random directions and as a whole
vector (relative L2 norm).
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

    # the library: FP32 forward window with checkpoints, hand-written reverse pass
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
    mass = sim.grain_mass.copy()
    sim.close()

    # FP64: the same window recorded, then frozen
    model = AT.model_from_config(cfg, sc.radius, mass)
    x0 = torch.tensor(start[:, :3], dtype=torch.float64, device="cuda")
    v0 = torch.tensor(start[:, 3:], dtype=torch.float64, device="cuda")
    sp0 = AT.springs_from_rows(n, *springs)
    th0 = torch.tensor([mu, e, k], dtype=torch.float64, device="cuda")
    m64 = model.mass

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
            print(f"theta[{a}]: library {g32_th[a]:.6e}  fp64 adjoint {g64_th[a]:.6e}  fd {fd:.6e}")
            assert _rel(g64_th[a], fd) < RTOL
            assert _rel(g32_th[a], fd) < RTOL
            assert _rel(g32_th[a], g64_th[a]) < RTOL
        # v0 in random directions
        for _ in range(3):
            dv = torch.tensor(rng.normal(size=(n, 3)), device="cuda")
            fd = float((loss64(v0 + h * dv, th0) - loss64(v0 - h * dv, th0)) / (2 * h))
            a32 = float((g32_v0 * dv).sum())
            a64 = float((g64_v0 * dv).sum())
            print(f"v0 direction: library {a32:.6e}  fp64 adjoint {a64:.6e}  fd {fd:.6e}")
            assert _rel(a64, fd) < RTOL
            assert _rel(a32, fd) < RTOL
    whole = float((g32_v0 - g64_v0).norm() / g64_v0.norm())
    print(f"v0 gradient, relative L2 difference library vs fp64 adjoint: {whole:.3e}")
    assert whole < RTOL
