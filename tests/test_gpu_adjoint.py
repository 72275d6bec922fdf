"""The reverse pass (wd_adjoint_record / wd_adjoint_backward / wd_deposit_vjp) against
central finite differences of the FP64 restatement (tests/adjoint_ref.py) with the
contact pattern of its base run frozen.

The adjoint runs in FP32 on the FP32 trajectory; the differences run in FP64 on the FP64
trajectory (which follows the oracle to 1e-6 m over these windows). Directional
derivatives must agree to 0.1% (measured on a B200: 1e-7 to 5e-5 relative).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from adjoint_ref import cic, run
from test_adjoint_ref import model_for, scene
from world_b200 import ParticleDynamics
from world_b200.adjoint import deposit, window

pytestmark = pytest.mark.gpu

RTOL = 1e-3


def _fd(f, h):
    return (f(h) - f(-h)) / (2.0 * h)


def _close(adj, fd):
    assert abs(adj - fd) <= RTOL * abs(fd) + 1e-12 * (1.0 + abs(fd)), (adj, fd)


@pytest.mark.parametrize("history", [True, False])
def test_window_adjoint_matches_finite_differences(history):
    cfg, st, rad, mass = scene(history, n=400, seed=5)
    ph = cfg.physics
    mu, e, k = float(ph.friction), float(ph.restitution), float(ph.normal_stiffness)
    steps, every = 30, 10
    sim = ParticleDynamics(cfg, state=st, radius=rad)
    sim.set_contact_params(mu, e, k)
    sim.adjoint_record(steps, every)
    rng = np.random.default_rng(7)
    wx = rng.normal(size=(sim.n, 3))
    wv = rng.normal(size=(sim.n, 3)) * 1e-3
    gx0, gv0, gth = sim.adjoint_backward(torch.tensor(wx, dtype=torch.float32, device="cuda"),
                                          torch.tensor(wv, dtype=torch.float32, device="cuda"))
    gx0 = gx0.cpu().double().numpy()
    gv0 = gv0.cpu().double().numpy()

    model = model_for(cfg, rad, mass)
    x0, v0 = st[:, :3].astype(np.float64), st[:, 3:].astype(np.float64)
    _, _, pat = run(model, x0, v0, mu, e, k, steps)

    def loss(x_, v_, mu_, e_, k_):
        xT, vT, _ = run(model, x_, v_, mu_, e_, k_, steps, pattern=pat)
        return float((wx * xT).sum() + (wv * vT).sum())

    dv = rng.normal(size=v0.shape)
    dx = rng.normal(size=x0.shape)
    _close(float((gv0 * dv).sum()), _fd(lambda h: loss(x0, v0 + h * dv, mu, e, k), 1e-6))
    _close(float((gx0 * dx).sum()), _fd(lambda h: loss(x0 + h * dx, v0, mu, e, k), 1e-9))
    _close(gth[0], _fd(lambda h: loss(x0, v0, mu + h, e, k), 1e-6))
    _close(gth[1], _fd(lambda h: loss(x0, v0, mu, e + h, k), 1e-6))
    _close(gth[2], _fd(lambda h: loss(x0, v0, mu, e, k + h), 1e-2))
    sim.close()


def test_backward_leaves_the_window_end_and_the_run_continues_unchanged():
    cfg, st, rad, _ = scene(True, n=300, seed=9)
    a = ParticleDynamics(cfg, state=st, radius=rad)
    b = ParticleDynamics(cfg, state=st, radius=rad)
    a.adjoint_record(25, 10)
    b.advance(25)
    end = a.get_state()
    np.testing.assert_array_equal(end, b.get_state())
    g = torch.ones((a.n, 3), device="cuda")
    a.adjoint_backward(g, g)
    np.testing.assert_array_equal(a.get_state(), end)
    assert a.time == b.time
    a.advance(20)
    b.advance(20)
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    assert a.grid_overflow_count() == b.grid_overflow_count()
    a.close(); b.close()


def test_deposit_vjp_matches_finite_differences():
    cfg, st, rad, mass = scene(True, n=300, seed=11)
    sim = ParticleDynamics(cfg, state=st, radius=rad)
    sim.advance(10)
    state = sim.get_state().reshape(-1, 6).astype(np.float64)
    x, v = state[:, :3], state[:, 3:]
    size = (cfg.density_grid_size_x, cfg.density_grid_size_y, cfg.density_grid_size_z)
    lo = [cfg.domain.x_min, cfg.domain.y_min, cfg.domain.z_min]
    hi = [cfg.domain.x_max, cfg.domain.y_max, cfg.domain.z_max]
    rng = np.random.default_rng(3)
    G = rng.normal(size=(4, *size))
    gx, gv = sim.deposit_vjp(torch.tensor(G.reshape(-1), dtype=torch.float32, device="cuda"))
    gx, gv = gx.cpu().double().numpy(), gv.cpu().double().numpy()
    m = mass.astype(np.float64)
    dx = rng.normal(size=x.shape)
    dv = rng.normal(size=v.shape)
    f = lambda xx, vv: float((G * cic(xx, vv, m, lo, hi, size)).sum())
    _close(float((gx * dx).sum()), _fd(lambda h: f(x + h * dx, v), 1e-9))
    _close(float((gv * dv).sum()), _fd(lambda h: f(x, v + h * dv), 1e-6))
    sim.close()


def test_autograd_density_loss_gradients():
    """loss = mean((rho_T - rho_target)^2) through window() and deposit(); the gradients
    in v0 and (mu, e, k_n) against FD of the same pipeline in FP64."""
    cfg, st, rad, mass = scene(True, n=300, seed=13)
    ph = cfg.physics
    mu, e, k = float(ph.friction), float(ph.restitution), float(ph.normal_stiffness)
    steps = 20
    size = (cfg.density_grid_size_x, cfg.density_grid_size_y, cfg.density_grid_size_z)
    lo = [cfg.domain.x_min, cfg.domain.y_min, cfg.domain.z_min]
    hi = [cfg.domain.x_max, cfg.domain.y_max, cfg.domain.z_max]
    m = mass.astype(np.float64)
    model = model_for(cfg, rad, mass)
    x0, v0 = st[:, :3].astype(np.float64), st[:, 3:].astype(np.float64)
    # target: the same window with mu = 0.4, e = 0.6
    xt, vt, _ = run(model, x0, v0, 0.4, 0.6, k, steps)
    target = cic(xt, vt, m, lo, hi, size)[0]

    sim = ParticleDynamics(cfg, state=st, radius=rad)
    tx0 = torch.tensor(st[:, :3], device="cuda", requires_grad=True)
    tv0 = torch.tensor(st[:, 3:], device="cuda", requires_grad=True)
    theta = torch.tensor([mu, e, k], dtype=torch.float64, requires_grad=True)
    x, v = window(sim, tx0, tv0, theta, steps, 10)
    grid = deposit(sim, x, v)
    loss = ((grid[0].double() - torch.tensor(target, device="cuda")) ** 2).mean()
    loss.backward()

    _, _, pat = run(model, x0, v0, mu, e, k, steps)

    def L(v_, mu_, e_, k_):
        xT, vT, _ = run(model, x0, v_, mu_, e_, k_, steps, pattern=pat)
        return float(((cic(xT, vT, m, lo, hi, size)[0] - target) ** 2).mean())

    assert abs(float(loss.detach()) - L(v0, mu, e, k)) < 1e-3 * L(v0, mu, e, k) + 1e-20
    rng = np.random.default_rng(5)
    dv = rng.normal(size=v0.shape)
    _close(float((tv0.grad.cpu().double().numpy() * dv).sum()), _fd(lambda h: L(v0 + h * dv, mu, e, k), 1e-6))
    g = theta.grad.numpy()
    _close(g[0], _fd(lambda h: L(v0, mu + h, e, k), 1e-6))
    _close(g[1], _fd(lambda h: L(v0, mu, e + h, k), 1e-6))
    _close(g[2], _fd(lambda h: L(v0, mu, e, k + h), 1e-2))
    sim.close()
