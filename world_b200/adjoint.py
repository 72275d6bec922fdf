"""torch.autograd over the DEM step: a window of semi-implicit Euler steps and the CIC
deposit as differentiable functions, with the library's hand-written reverse pass.

    sim = ParticleDynamics(cfg, state=state, radius=radius)
    theta = torch.tensor([mu, e, k_n], dtype=torch.float64, requires_grad=True)
    v0 = torch.tensor(state[:, 3:], device="cuda", requires_grad=True)
    x, v = window(sim, x0, v0, theta, steps=200, checkpoint_every=20)
    grid = deposit(sim, x, v)                 # (4, nx, ny, nz): mass, momentum
    loss = ((grid[0] - target) ** 2).mean()
    loss.backward()                            # v0.grad, theta.grad

The reference has no derivatives; the contact set and the clamp / stick-slip / viscous
branches of every step are those the forward took (world_b200/csrc/wd_adjoint.cu).
A window starts from (x0, v0) and the handle's current tangential springs (its
history rows); set them (set_history) before evaluating the same window again.
"""
from __future__ import annotations

import numpy as np
import torch


class _Window(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, theta, sim, steps, checkpoint_every):
        th = theta.detach().double().cpu().numpy()
        sim.set_contact_params(float(th[0]), float(th[1]), float(th[2]))
        state = torch.cat([x0.detach().float(), v0.detach().float()], dim=1).to("cuda").contiguous()
        sim.set_state_tensor(state.reshape(-1))
        sim.adjoint_record(int(steps), int(checkpoint_every))
        out = sim.state_tensor().reshape(-1, 6)
        ctx.sim = sim
        ctx.theta_dtype = theta.dtype
        ctx.theta_device = theta.device
        return out[:, :3].clone(), out[:, 3:].clone()

    @staticmethod
    def backward(ctx, gx, gv):
        gx0, gv0, gth = ctx.sim.adjoint_backward(gx, gv)
        gtheta = torch.tensor(gth, dtype=ctx.theta_dtype, device=ctx.theta_device)
        return gx0, gv0, gtheta, None, None, None


class _Deposit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, v, sim):
        ctx.sim = sim
        sim.compute_density_grid()
        g = torch.from_numpy(sim.host_density_grid.copy()).to("cuda")
        return g.reshape(4, sim.density_grid_size_x, sim.density_grid_size_y,
                         sim.density_grid_size_z)

    @staticmethod
    def backward(ctx, ggrid):
        gx, gv = ctx.sim.deposit_vjp(ggrid.reshape(-1))
        return gx, gv, None


def window(sim, x0: torch.Tensor, v0: torch.Tensor, theta: torch.Tensor, steps: int,
           checkpoint_every: int = 20):
    """(x, v) after `steps` steps from (x0, v0) with contact parameters theta =
    (mu, restitution, k_n); differentiable in x0, v0 and theta."""
    return _Window.apply(x0, v0, theta, sim, steps, checkpoint_every)


def deposit(sim, x: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """The CIC field (4, nx, ny, nz) of the simulation's current state, which must be
    (x, v) -- the output of window(); differentiable in x and v."""
    return _Deposit.apply(x, v, sim)
