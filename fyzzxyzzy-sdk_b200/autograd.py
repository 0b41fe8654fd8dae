"""torch.autograd binding of the differentiable rollout (a thin test and
convenience layer over fyzz_b200_rollout_*; the adjoint itself is the
library's CUDA code).

    c, v, w = rollout(world, v0, w0, mass, friction, steps=128, every=16)

runs `steps` steps from the world's current poses with initial velocities
(v0, w0) and returns the final mass-frame centres and velocities.  `mass`
(per body) and `friction` (per shape, static = dynamic) must hold the
world's current values: they are inputs so that autograd returns their
gradients.  Backward calls fyzz_b200_rollout_backward.
"""
from __future__ import annotations

import numpy as np
import torch


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v0, w0, mass, friction, world, steps: int, every: int, dt: float):
        v6 = torch.cat([v0.detach(), w0.detach()], 1).to(torch.float32).cpu().numpy()
        world.write_velocities(np.ascontiguousarray(v6))
        world.rollout_begin(steps, every)
        world.rollout_forward(dt)
        c, _ = world.read_mass_frames()
        st = world.read_bodies()
        ctx.world = world
        ctx.dtype = v0.dtype
        return (torch.from_numpy(c).to(v0.dtype), torch.from_numpy(st[:, 3:6].copy()).to(v0.dtype),
                torch.from_numpy(st[:, 10:13].copy()).to(v0.dtype))

    @staticmethod
    def backward(ctx, gc, gv, gw):
        as_np = lambda g: None if g is None else g.detach().to(torch.float32).cpu().numpy()
        g = ctx.world.rollout_backward(as_np(gc), None, as_np(gv), as_np(gw))
        t = lambda x: torch.from_numpy(np.asarray(x)).to(ctx.dtype)
        return (t(g["v0"]), t(g["w0"]), t(g["mass"]), t(g["static_friction"] + g["dynamic_friction"]),
                None, None, None, None)


def rollout(world, v0, w0, mass, friction, steps: int, every: int, dt: float = 1.0 / 120.0):
    return Rollout.apply(v0, w0, mass, friction, world, steps, every, dt)
