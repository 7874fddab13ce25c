"""Headless stress run on the GPU, a drop-in for the reference's
stress_test_blocks example (examples/stress_test_blocks/main.cpp).

    python -m dyphur_b200.run [out_prefix] [n_frames] [--grid NX NY NZ]
                              [--spacing S] [--jitter J] [--profile]
                              [--workload blocks|pile|batch] [--mode M]
                              [--start-frame F] [--smem-cap B] [--teams T]
                              [--autotune FRAMES] [--adjoint EVERY]

Writes <prefix>.scene, <prefix>.trajectory (poses every other frame),
<prefix>.metrics.json and <prefix>.golden exactly as the example does. The
default scene is the example's own: 8 x 16 x 8 boxes of half extent 0.4 m at
1.0 m spacing, no jitter, on a ground plate, 300 frames at 60 Hz.

--profile prints the per-stage milliseconds per frame over the frames after
30 warm-up frames (the example's --profile table), timed by CUDA events
recorded inside the captured frames instead of host fences.
--start-frame F steps F frames untimed and writes nothing before the run:
with `ncu -k regex:<kernel> -s F -c 1` it captures frame F's launch of a
kernel that runs once per frame.
--adjoint EVERY runs one differentiable rollout of n_frames (checkpoints every
EVERY frames) and its backward pass instead, loss = squared distance of the
boxes to the scenes' targets (the push workload), and prints both times; the
backward pass runs one record and one reverse launch per frame, last frame
first, so `ncu -k regex:scene_frame_reverse -s F -c 1` captures frame
n_frames - 1 - F's reverse launch.
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np


def parse(argv=None):
    ap = argparse.ArgumentParser(prog="python -m dyphur_b200.run")
    ap.add_argument("prefix", nargs="?", default="stress_test_blocks")
    ap.add_argument("n_frames", nargs="?", type=int, default=300)
    ap.add_argument("--grid", nargs=3, type=int, default=(8, 16, 8), metavar=("NX", "NY", "NZ"))
    ap.add_argument("--spacing", type=float, default=1.0)
    ap.add_argument("--jitter", type=float, default=0.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--workload", default="blocks", choices=["blocks", "pile", "batch", "push"])
    ap.add_argument("--bodies", type=int, default=65536, help="pile: dynamic bodies")
    ap.add_argument("--scenes", type=int, default=4096, help="batch, push: scenes")
    ap.add_argument("--adjoint", type=int, default=0, metavar="EVERY",
                    help="one rollout of n_frames and its backward pass, checkpoints every EVERY frames")
    ap.add_argument("--mode", default="reference", choices=["reference", "sequential", "colored"])
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--start-frame", type=int, default=0)
    ap.add_argument("--no-output", action="store_true", help="write no files")
    ap.add_argument("--smem-cap", type=int, default=None,
                    help="batch: shared memory cap per block of the fused frame (bytes; 0 = what it needs)")
    ap.add_argument("--teams", type=int, default=None, choices=[0, 1, 2],
                    help="batch: 0 every scene a block, 1 small scenes one per warp, 2 also mid-size on two warps")
    ap.add_argument("--register-blocks", type=int, default=0, choices=[0, 4, 5, 6],
                    help="batch: register budget of the fused frame kernel (resident blocks per SM)")
    ap.add_argument("--autotune", type=int, default=0, metavar="FRAMES",
                    help="batch: autotune the fused frame on FRAMES frames (after --start-frame) first")
    ap.add_argument("--rays", type=int, default=0, metavar="N",
                    help="after the run, cast N seeded rays at the bodies through the last frame's tree")
    return ap.parse_args(argv)


def build_scene(args):
    from . import scenes
    if args.workload == "pile":
        return scenes.random_pile(args.bodies, seed=args.seed)
    if args.workload == "batch":
        return scenes.batch(args.scenes, 8, 256, seed=args.seed)
    if args.workload == "push":
        return scenes.push(args.scenes, seed=args.seed)
    nx, ny, nz = args.grid
    return scenes.stress_blocks(spacing=args.spacing, jitter=args.jitter, seed=args.seed, grid=(nx, ny, nz))


def profile(world, scene, frames: int, warm: int = 30) -> None:
    """Per-stage ms per frame (integrate, broadphase, narrowphase, solver);
    for a fused batched world, the frame's wall time and its phases' share
    of the scenes' summed work time."""
    import torch
    from . import capi
    names = ("integrate", "build_and_query", "narrowphase", "solve (XPBD)")
    fb = world.bodies.fbuf
    init = fb.clone()
    world.step(warm)
    start = fb.clone()
    try:
        world.phase_timing(True)
    except capi.DyphError:
        pass
    else:
        world.capture_episode(frames, 4)
        world.run_episode()
        torch.cuda.synchronize()
        ms = float(world.probe_ms().mean())
        ph = world.phase_ns().astype(np.float64)
        world.phase_timing(False)
        fb.copy_(init)
        labels = ("stage+integrate+boxes", "pair search", "narrowphase", "solve set-up", "sweep+renorm",
                  "write-back")
        print(f"-- Fused frame: {ms:.3f} ms per frame over {frames} warm frames ({scene.n_scenes} scenes, "
              f"{scene.n_bodies} bodies); phases, share of the scenes' summed work time --")
        for name, v in zip(labels, ph):
            print(f"  {name:<22} {100.0 * v / ph.sum():5.1f}%   ({v / frames / 1e3:10.1f} us summed per frame)")
        return
    rows = []
    for stage in range(4):
        fb.copy_(start)
        world.capture_episode(frames, stage)
        world.run_episode()
        torch.cuda.synchronize()
        rows.append(float(world.probe_ms().mean()))
    fb.copy_(init)
    total = sum(rows)
    print(f"-- Per-stage avg over {frames} warm frames ({scene.n_bodies} bodies) --")
    for name, ms in zip(names, rows):
        print(f"  {name:<16} {ms:8.3f} ms   {100.0 * ms / total:5.1f}%")
    print(f"  {'TOTAL':<16} {total:8.3f} ms   ({1000.0 / total:.1f} fps, stage-summed)")


def cast_rays(world, scene, n_rays: int, seed: int = 9) -> None:
    """N rays from random points of the scene's box aimed near random bodies,
    through the last frame's tree (ray_query); prints hits and rays/s."""
    import torch
    rng = np.random.default_rng(seed)
    st = world.state()
    lo, hi = scene.bounds[0, :3], scene.bounds[0, 3:]
    target = st[:3].T[rng.integers(0, scene.n_bodies, n_rays)] + rng.normal(0.0, 0.3, (n_rays, 3))
    origin = rng.uniform(lo, hi, (n_rays, 3))
    rays = torch.from_numpy(np.concatenate([origin, target - origin, np.full((n_rays, 1), 1e9)], 1)
                            .astype(np.float32)).cuda()
    world.ray_query(rays)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    t, body = world.ray_query(rays)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    hits = int((body != -1).sum())
    print(f"rays: {n_rays} cast, {hits} hit, {ms:.3f} ms ({n_rays / ms / 1e3:.1f} M rays/s)")


def adjoint_run(world, scene, frames: int, every: int) -> None:
    """One differentiable rollout (sequential order) and its backward pass:
    loss = sum over the dynamic bodies of |x_final - target|^2 (targets of the
    push workload; the origin otherwise). Prints the forward and backward
    milliseconds and the gradient norm."""
    import torch
    from .autograd import rollout
    n = scene.n_bodies
    target = getattr(scene, "targets", None)
    tgt = torch.zeros((n, 3), device="cuda") if target is None else torch.from_numpy(target).cuda()
    dyn = torch.from_numpy((scene.mass > 0).astype(np.float32)).cuda()
    vel = world.initial[7:10, :n].T.clone().requires_grad_(True)
    ang = world.initial[10:13, :n].T.clone().requires_grad_(True)
    im = world.bodies.fbuf[13, :n].clone().requires_grad_(True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    final = rollout(world, vel, ang, im, frames, every=every)
    ev[1].record()
    ((((final[:3].T - tgt) ** 2).sum(1)) * dyn).sum().backward()
    ev[2].record()
    torch.cuda.synchronize()
    g = float(torch.linalg.vector_norm(torch.cat([vel.grad.ravel(), ang.grad.ravel(), im.grad.ravel()])))
    print(f"adjoint: {frames} frames, checkpoints every {every}: forward {ev[0].elapsed_time(ev[1]):.3f} ms, "
          f"backward {ev[1].elapsed_time(ev[2]):.3f} ms, |gradient| {g:.6g}; reverse kernel layout "
          f"{world.adjoint_config()}")


def main(argv=None) -> int:
    import torch

    from . import capi, device, formats

    args = parse(argv)
    mode = {"reference": capi.SOLVER_REFERENCE, "sequential": capi.SOLVER_SEQUENTIAL,
            "colored": capi.SOLVER_COLORED}[args.mode]
    scene = build_scene(args)
    n = scene.n_bodies
    world = device.World(scene, mode=mode)
    if args.smem_cap is not None or args.teams is not None or args.register_blocks:
        world.set_fused_config(args.smem_cap or 0, 2 if args.teams is None else args.teams, args.register_blocks)
    if args.autotune:
        init = world.bodies.fbuf.clone()
        world.step(args.start_frame)
        cfg = world.autotune(args.autotune)
        world.bodies.fbuf.copy_(init)
        torch.cuda.synchronize()
        print(f"fused frame configuration: {cfg}")
    if args.adjoint:
        if mode != capi.SOLVER_SEQUENTIAL:
            print("--adjoint needs --mode sequential", file=sys.stderr)
            return 2
        adjoint_run(world, scene, args.n_frames, args.adjoint)
        return 0
    if args.start_frame:
        world.step(args.start_frame)
        world.step(args.n_frames)
        torch.cuda.synchronize()
        st = world.stats()
        print(f"stepped {args.start_frame} + {args.n_frames} frames, status {st['status']}, last frame "
              f"{st['last_pairs']} candidate pairs, {st['last_contacts']} contacts, {n} bodies")
        if args.rays:
            cast_rays(world, scene, args.rays)
        return 0
    if args.profile:
        profile(world, scene, args.n_frames)
        return 0
    if not args.no_output:
        formats.write_scene_set(args.prefix, scene)
    records = formats.trajectory_records(args.n_frames)
    traj = torch.empty((max(records, 1), n, 7), dtype=torch.float32).pin_memory()
    world.set_trajectory(traj, 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    world.step(args.n_frames)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    world.set_trajectory(None)
    st = world.stats()
    h = world.hash()
    if not args.no_output:
        formats.write_trajectory(args.prefix, args.n_frames, traj.numpy()[:records])
        formats.write_golden(args.prefix, h)
        formats.write_metrics(args.prefix, n, args.n_frames, scene.dt, wall, float(st["last_contacts"]))
    over = st["peak_pairs"] > world.desc.max_pairs or st["peak_contacts"] > world.desc.max_contacts
    print(f"Peak usage: pairs {st['peak_pairs']}/{world.desc.max_pairs}, contacts "
          f"{st['peak_contacts']}/{world.desc.max_contacts}" + (" -- CAPACITY OVERFLOW" if over else ""))
    fps = args.n_frames / wall if wall > 0 else 0.0
    print(f"Completed {args.n_frames} frames in {wall:.3f}s ({fps:.1f} fps, {fps / 60.0:.2f}x realtime)")
    print(f"Hash: {h:016x}")
    if not args.no_output:
        print(f"Wrote: {args.prefix}.scene  {args.prefix}.trajectory  {args.prefix}.metrics.json  "
              f"{args.prefix}.golden")
    return 0 if not over and st["status"] == 0 else 1


if __name__ == "__main__":
    sys.exit(main())
