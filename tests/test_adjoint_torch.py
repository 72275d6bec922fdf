"""The torch FP64 restatement (tests/adjoint_torch.py) against the numpy one
(tests/adjoint_ref.py, itself pinned to the oracle), its frozen replay, and its autograd
adjoint against central differences. CPU only (torch float64 on the host)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import adjoint_ref
import adjoint_torch as AT
from test_adjoint_ref import model_for, scene


def _setup(n=400, seed=5):
    cfg, st, rad, mass = scene(True, n=n, seed=seed)
    model = AT.model_from_config(cfg, rad, mass, device="cpu")
    ph = cfg.physics
    params = (float(ph.friction), float(ph.restitution), float(ph.normal_stiffness))
    empty = (torch.zeros(0, dtype=torch.int64), torch.zeros((0, 3), dtype=torch.float64))
    return cfg, st, rad, mass, model, params, empty


def test_torch_restatement_equals_numpy_restatement():
    cfg, st, rad, mass, model, (mu, e, k), empty = _setup()
    steps = 30
    xn, vn, pat = adjoint_ref.run(model_for(cfg, rad, mass), st[:, :3], st[:, 3:], mu, e, k, steps)
    x0 = torch.tensor(st[:, :3], dtype=torch.float64)
    v0 = torch.tensor(st[:, 3:], dtype=torch.float64)
    xt, vt, rec = AT.run(model, x0, v0, empty, torch.tensor(mu, dtype=torch.float64),
                         torch.tensor(e, dtype=torch.float64), torch.tensor(k, dtype=torch.float64),
                         steps)
    assert sum(p.pairs[0].size for p in pat) > 1000
    assert sum(int(r["pairs"][0].numel()) for r in rec) == sum(p.pairs[0].size for p in pat)
    np.testing.assert_allclose(xt.numpy(), xn, rtol=0, atol=1e-12)
    np.testing.assert_allclose(vt.numpy(), vn, rtol=0, atol=1e-9 * np.abs(vn).max())
    # the frozen replay reproduces the run
    x2, v2, _ = AT.run(model, x0, v0, empty, torch.tensor(mu, dtype=torch.float64),
                       torch.tensor(e, dtype=torch.float64), torch.tensor(k, dtype=torch.float64),
                       steps, pattern=rec)
    assert torch.equal(x2, xt) and torch.equal(v2, vt)


def test_torch_adjoint_matches_central_differences():
    cfg, st, rad, mass, model, (mu, e, k), empty = _setup(n=300, seed=13)
    steps = 20
    x0 = torch.tensor(st[:, :3], dtype=torch.float64)
    v0 = torch.tensor(st[:, 3:], dtype=torch.float64)
    th = torch.tensor([mu, e, k], dtype=torch.float64)
    _, _, pat = AT.run(model, x0, v0, empty, th[0], th[1], th[2], steps)
    rng = np.random.default_rng(1)
    wx = torch.tensor(rng.normal(size=(model.n, 3)))
    wv = torch.tensor(rng.normal(size=(model.n, 3)) * 1e-3)

    def loss(v_, th_):
        xT, vT, _ = AT.run(model, x0, v_, empty, th_[0], th_[1], th_[2], steps, pattern=pat)
        return (wx * xT).sum() + (wv * vT).sum()

    tv = v0.clone().requires_grad_(True)
    tth = th.clone().requires_grad_(True)
    loss(tv, tth).backward()
    dv = torch.tensor(rng.normal(size=(model.n, 3)))
    fd = (loss(v0 + 1e-6 * dv, th) - loss(v0 - 1e-6 * dv, th)) / 2e-6
    assert float((tv.grad * dv).sum()) == pytest.approx(float(fd), rel=1e-6)
    for a, h in ((0, 1e-6), (1, 1e-6), (2, 1e-2)):
        dth = torch.zeros(3, dtype=torch.float64)
        dth[a] = h
        fd = (loss(v0, th + dth) - loss(v0, th - dth)) / (2 * h)
        assert float(tth.grad[a]) == pytest.approx(float(fd), rel=1e-6, abs=1e-12)


def test_torch_cic_matches_numpy_cic():
    rng = np.random.default_rng(0)
    x = rng.uniform(-0.9, 0.9, (60, 3))
    v = rng.normal(size=(60, 3))
    m = rng.uniform(0.5, 2.0, 60)
    m[3] = 0.0
    lo, hi, size = [-1.0] * 3, [1.0] * 3, (8, 9, 10)
    want = adjoint_ref.cic(x, v, m, lo, hi, size)
    got = AT.cic(torch.tensor(x), torch.tensor(v), torch.tensor(m), lo, hi, size)
    np.testing.assert_allclose(got.numpy(), want, rtol=1e-12, atol=1e-12)


def test_adjoint_along_a_trajectory_equals_autograd_through_the_window():
    """Chaining per-step vector-Jacobian products at the recorded states (what the C4 test
    does along the library's trajectory) equals autograd through the frozen window when
    the states are the window's own."""
    cfg, st, rad, mass, model, (mu, e, k), empty = _setup(n=300, seed=13)
    steps = 15
    x0 = torch.tensor(st[:, :3], dtype=torch.float64)
    v0 = torch.tensor(st[:, 3:], dtype=torch.float64)
    th = torch.tensor([mu, e, k], dtype=torch.float64)
    rng = np.random.default_rng(2)
    wx = torch.tensor(rng.normal(size=(model.n, 3)))
    wv = torch.tensor(rng.normal(size=(model.n, 3)) * 1e-3)
    _, _, pat = AT.run(model, x0, v0, empty, th[0], th[1], th[2], steps)
    tv = v0.clone().requires_grad_(True)
    tth = th.clone().requires_grad_(True)
    xT, vT, _ = AT.run(model, x0, tv, empty, tth[0], tth[1], tth[2], steps, pattern=pat)
    ((wx * xT).sum() + (wv * vT).sum()).backward()
    traj, sprs = AT.record_trajectory(model, x0, v0, empty, th, steps)
    gv, _, gth = AT.adjoint_along(model, traj, sprs, th,
                                  lambda x, v: (wx * x).sum() + (wv * v).sum())
    assert sum(int(s[0].numel()) for s in sprs) > 500        # springs carried through
    np.testing.assert_allclose(gv.numpy(), tv.grad.numpy(), rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(gth.numpy(), tth.grad.numpy(), rtol=1e-9, atol=0)


def test_adjoint_along_in_float32_stays_near_float64():
    """The float32 evaluation of the chain (the C4 test's measure of what FP32 arithmetic
    does to a window's adjoint) runs in float32 throughout and, on a short window, lands
    near the float64 one."""
    cfg, st, rad, mass, model, (mu, e, k), empty = _setup(n=300, seed=13)
    steps = 15
    x0 = torch.tensor(st[:, :3], dtype=torch.float64)
    v0 = torch.tensor(st[:, 3:], dtype=torch.float64)
    th = torch.tensor([mu, e, k], dtype=torch.float64)
    rng = np.random.default_rng(3)
    wx = torch.tensor(rng.normal(size=(model.n, 3)))
    wv = torch.tensor(rng.normal(size=(model.n, 3)) * 1e-3)
    traj, sprs = AT.record_trajectory(model, x0, v0, empty, th, steps)
    loss = lambda x, v: (wx * x.double()).sum() + (wv * v.double()).sum()  # noqa: E731
    gv, _, gth = AT.adjoint_along(model, traj, sprs, th, loss)
    m32 = AT.model_as(model, torch.float32)
    gv32, _, gth32 = AT.adjoint_along(m32, [t.float() for t in traj],
                                      [(kk, xi.float()) for kk, xi in sprs], th.float(), loss)
    assert gv32.dtype == torch.float32 and gth32.dtype == torch.float32
    assert float((gv32.double() - gv).norm() / gv.norm()) < 1e-4
    np.testing.assert_allclose(gth32.double().numpy(), gth.numpy(), rtol=1e-3)
