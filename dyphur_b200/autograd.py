"""Gradients through the frame step: a torch.autograd.Function over the
library's rollout and its hand-written adjoint (dyph_world_rollout /
dyph_world_rollout_backward).

    world = device.World(scenes.push(256), mode=capi.SOLVER_SEQUENTIAL)
    vel = torch.tensor(..., requires_grad=True)       # (n, 3) initial velocities
    ang = torch.tensor(..., requires_grad=True)       # (n, 3) initial spins
    inv_mass = torch.tensor(..., requires_grad=True)  # (n,) inverse masses
    final = rollout(world, vel, ang, inv_mass, frames=120, every=10)  # (13, n)
    loss = ((final[:3].T[boxes] - targets[boxes]) ** 2).sum(-1).mean()
    loss.backward()

The world (dyphur_b200.device.World or dyphur_py.World) must be a batched
world whose frames run fused (dyph_world_set_scenes on scenes that fit one
thread block). Positions and rotations start from the
world's initial state (`World.initial`). The contact set and every branch of
each frame are held fixed in the backward pass; static bodies get no gradient.
"""
from __future__ import annotations

import torch


def _rows(world):
    """(20, capacity) float32 CUDA tensor over the world's body rows, no copy."""
    r = world.device_rows()
    return r if isinstance(r, torch.Tensor) else torch.as_tensor(r, device="cuda")


class Rollout(torch.autograd.Function):
    """final_state (13, n) = frames of the world's step from (pos, rot) of
    `initial`, velocities `vel`, spins `ang` and inverse masses `inv_mass`.

    `world` is a dyphur_b200.device.World or a dyphur_py.World: both give
    device_rows(), count(), rollout_raw() and rollout_backward_raw()."""

    @staticmethod
    def forward(ctx, vel, ang, inv_mass, world, frames: int, every: int, initial):
        n = world.count()
        fb = _rows(world)
        with torch.no_grad():
            fb[:13, :n] = initial[:13, :n]
            fb[7:10, :n] = vel.detach().T.to(fb.dtype)
            fb[10:13, :n] = ang.detach().T.to(fb.dtype)
            fb[13, :n] = inv_mass.detach().to(fb.dtype)
        n_ckpt = (frames + every - 1) // every
        ckpt = torch.empty((n_ckpt, 13, n), dtype=torch.float32, device=fb.device)
        stream = torch.cuda.current_stream()
        world.rollout_raw(frames, every, ckpt.data_ptr(), stream.cuda_stream)
        out = fb[:13, :n].clone()
        ctx.world, ctx.frames, ctx.every = world, frames, every
        ctx.save_for_backward(ckpt, inv_mass)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        ckpt, inv_mass = ctx.saved_tensors
        world = ctx.world
        n = world.count()
        fb = _rows(world)
        with torch.no_grad():
            fb[13, :n] = inv_mass.detach().to(fb.dtype)
        g_final = grad_out.detach().to(torch.float32).contiguous()
        g_init = torch.empty((13, n), dtype=torch.float32, device=fb.device)
        g_im = torch.empty(n, dtype=torch.float32, device=fb.device)
        stream = torch.cuda.current_stream()
        world.rollout_backward_raw(ctx.frames, ctx.every, ckpt.data_ptr(), g_final.data_ptr(), g_init.data_ptr(),
                                   g_im.data_ptr(), stream.cuda_stream)
        return g_init[7:10].T.contiguous(), g_init[10:13].T.contiguous(), g_im, None, None, None, None


def rollout(world, vel, ang, inv_mass, frames: int, every: int = 10, initial=None):
    """Differentiable rollout of `frames` frames (checkpoint every `every`
    frames); returns the final state (13, n): pos xyz, rot wxyz, vel xyz, ang xyz.
    `initial` defaults to the world's state at creation."""
    if initial is None:
        r = world.initial_rows()
        initial = r if isinstance(r, torch.Tensor) else torch.as_tensor(r, device="cuda")
    return Rollout.apply(vel, ang, inv_mass, world, frames, every, initial)
