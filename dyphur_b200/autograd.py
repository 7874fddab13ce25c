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

The world must be a batched world whose frames run fused (dyph_world_set_scenes
on scenes that fit one thread block). Positions and rotations start from the
world's initial state (`World.initial`). The contact set and every branch of
each frame are held fixed in the backward pass; static bodies get no gradient.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import capi
from .capi import check


class Rollout(torch.autograd.Function):
    """final_state (13, n) = frames of the world's step from (pos, rot) of
    `initial`, velocities `vel`, spins `ang` and inverse masses `inv_mass`."""

    @staticmethod
    def forward(ctx, vel, ang, inv_mass, world, frames: int, every: int, initial):
        n = world.bodies.n
        fb = world.bodies.fbuf
        with torch.no_grad():
            fb[:13, :n] = initial[:13, :n]
            fb[7:10, :n] = vel.detach().T.to(fb.dtype)
            fb[10:13, :n] = ang.detach().T.to(fb.dtype)
            fb[13, :n] = inv_mass.detach().to(fb.dtype)
        n_ckpt = (frames + every - 1) // every
        ckpt = torch.empty((n_ckpt, 13, n), dtype=torch.float32, device=fb.device)
        stream = torch.cuda.current_stream()
        check(capi.lib().dyph_world_rollout(world.h, frames, every, ckpt.data_ptr(), stream.cuda_stream),
              "dyph_world_rollout")
        out = fb[:13, :n].clone()
        ctx.world, ctx.frames, ctx.every = world, frames, every
        ctx.save_for_backward(ckpt, inv_mass)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        ckpt, inv_mass = ctx.saved_tensors
        world = ctx.world
        n = world.bodies.n
        fb = world.bodies.fbuf
        with torch.no_grad():
            fb[13, :n] = inv_mass.detach().to(fb.dtype)
        g_final = grad_out.detach().to(torch.float32).contiguous()
        g_init = torch.empty((13, n), dtype=torch.float32, device=fb.device)
        g_im = torch.empty(n, dtype=torch.float32, device=fb.device)
        stream = torch.cuda.current_stream()
        check(capi.lib().dyph_world_rollout_backward(world.h, ctx.frames, ctx.every, ckpt.data_ptr(),
                                                     g_final.data_ptr(), g_init.data_ptr(), g_im.data_ptr(),
                                                     stream.cuda_stream), "dyph_world_rollout_backward")
        return g_init[7:10].T.contiguous(), g_init[10:13].T.contiguous(), g_im, None, None, None, None


def rollout(world, vel, ang, inv_mass, frames: int, every: int = 10, initial=None):
    """Differentiable rollout of `frames` frames (checkpoint every `every`
    frames); returns the final state (13, n): pos xyz, rot wxyz, vel xyz, ang xyz."""
    if initial is None:
        initial = world.initial
    return Rollout.apply(vel, ang, inv_mass, world, frames, every, initial)
