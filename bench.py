#!/usr/bin/env python3
"""Frame-step benchmark (body-steps/s) on B200.

Workload: the large single-scene stress — 65536 bodies (70 % boxes with half
extents U[0.1, 0.5] m, 30 % spheres with r U[0.1, 0.4] m, density 500 kg/m^3)
dropped from a 40 m cube onto an 80 x 1 x 80 m ground, 600 frames at 60 Hz,
fp32, synthetic seeded input. One step = one 600-frame episode from the
initial state (the state is reset at the start of every step), replayed as one
CUDA graph through the library's world API.

  value  device-resident body-steps/s: the initial state is already in HBM.
  e2e    the same through the C-ABI world with host buffers: every step uploads
         the bodies from pinned host memory and downloads the final state.

Multi-GPU (torchrun): replicas only — each rank simulates its own scene, no
collective on the data path; the timed region is the max over ranks.
`--impl reference` times the reference's own frame-step sources (built on the
host SYCL shim with OpenMP) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOAD = ("large single-scene stress: 65536 bodies (70% boxes half-extent U[0.1,0.5] m, 30% spheres "
            "r U[0.1,0.4] m, 500 kg/m^3, random rotations, v N(0,0.5) m/s) in a 40 m cube over an "
            "80x1x80 m ground, 600 frames at 60 Hz, fp32")
METRIC = "body-steps/s"
STAGES = ("integrate", "broadphase", "narrowphase", "solver")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="single", choices=["single", "batch"],
                    help="single: the 65k-body pile; batch: 4096 independent scenes of 8-256 bodies")
    ap.add_argument("--scenes", type=int, default=4096)
    ap.add_argument("--frames", type=int, default=None)
    ap.add_argument("--start-frame", type=int, default=0,
                    help="step the pile this many frames (untimed) before recording the episode")
    ap.add_argument("--bodies", type=int, default=65536)
    ap.add_argument("--probe-stage", default="solver", choices=STAGES)
    ap.add_argument("--mode", default="reference", choices=["reference", "sequential", "colored"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-worker", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-frames", type=int, default=60)
    return ap.parse_args()


# ── CPU baseline (reference build or oracle port), run in a child process ────

def cpu_worker(which: str, bodies: int, frames: int) -> None:
    from dyphur_b200 import scenes
    from oracle import oracle
    s = scenes.random_pile(bodies)
    w = oracle.World(s, which)
    t0 = time.perf_counter()
    rc = w.step(frames)
    dt = time.perf_counter() - t0
    print(json.dumps({"rc": rc, "seconds": dt, "frames": frames, "bodies": s.n_bodies}))


def cpu_baseline(bodies: int, frames: int) -> dict | None:
    from oracle import oracle
    which = "ref" if oracle.ref_available() else "oracle"
    cores = os.cpu_count() or 1
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(cores if which == "ref" else 1)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", which, "--bodies", str(bodies),
           "--cpu-frames", str(frames)]
    try:
        out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900, check=True)
        r = json.loads(out.stdout.strip().splitlines()[-1])
    except Exception as e:  # the baseline is reported, not required
        print(f"cpu baseline failed: {e}", file=sys.stderr)
        return None
    return {"value": r["bodies"] * r["frames"] / r["seconds"], "unit": METRIC,
            "cores": cores if which == "ref" else 1, "kind": "reference" if which == "ref" else "port",
            "sample": f"frames 0-{frames - 1} of the same 600-frame episode ({r['seconds']:.1f} s, "
                      f"{'reference sources, OpenMP' if which == 'ref' else 'C oracle, 1 thread'})"}


# ── clocks sampler ───────────────────────────────────────────────────────────

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self) -> dict | None:
        if not self.p:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ── algorithmic bytes per stage launch (per frame) ──────────────────────────

def stage_bytes(stage: str, n: int, pairs: np.ndarray, contacts: np.ndarray) -> np.ndarray:
    """Compulsory bytes of one frame's stage: each input read once, each output
    written once (per body / pair / contact figures of the frame-step data)."""
    p = pairs.astype(np.float64)
    c = contacts.astype(np.float64)
    if stage == "integrate":
        return np.full_like(p, 100.0 * n)
    if stage == "broadphase":
        return 160.0 * n + 8.0 * p
    if stage == "narrowphase":
        return 72.0 * p + 36.0 * c
    return 300.0 * c + 32.0 * n  # solver: contact rows + both bodies read/written, renormalise


def kernels_per_frame(n: int, n_scenes: int = 1) -> int:
    """Library kernels one frame launches (matches the ncu launch list in profiles/)."""
    if n_scenes > 1:  # (scene << 30 | code) keys: histogram + one pass per 8 key bits, + scene ranges
        key_bits = 30 + max(1, (n_scenes - 1).bit_length())
        sort = (1 if n <= 4096 else 1 + (key_bits + 7) // 8) + 1
    else:
        sort = 1 if n <= 4096 else 5  # one-block sort, or histogram + 4 onesweep passes
    # integrate, morton, sort, build, finalize, pair find (two passes), pair write, narrowphase,
    # solver (dataflow, round-synchronous, sequential: two of them return at once), stats
    return 1 + 1 + sort + 1 + 1 + 2 + 1 + 1 + 3 + 1


def peaks() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(stage: str, mean_algorithmic_bytes: float):
    """DRAM bytes per launch of the stage, from the committed ncu capture
    (profiles/traffic.json), scaled from the captured launch's units to the
    episode's mean launch by the ratio of algorithmic bytes."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            rec = json.load(f).get(stage)
        return float(rec["dram_bytes"]) * mean_algorithmic_bytes / float(rec["algorithmic_bytes"])
    except Exception:
        return None


def max_over_ranks(values, device="cpu"):
    """Element-wise max of per-rank timings over the process group (the
    slowest rank sets a multi-GPU step's time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    from dyphur_b200 import capi, device, scenes

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    mode = {"reference": capi.SOLVER_REFERENCE, "sequential": capi.SOLVER_SEQUENTIAL,
            "colored": capi.SOLVER_COLORED}[args.mode]
    if args.workload == "batch":
        # independent scenes in one world; sequential order keeps each scene exact
        scene = scenes.batch(args.scenes, 8, 256, seed=3 + rank)
        if args.mode == "reference":
            mode = capi.SOLVER_SEQUENTIAL
            args.mode = "sequential"
    else:
        scene = scenes.random_pile(args.bodies, seed=2 + rank)  # replicas: one scene per rank
    n = scene.n_bodies
    w = device.World(scene, mode=mode)
    if args.start_frame > 0:
        w.step(args.start_frame)
    stage_idx = STAGES.index(args.probe_stage)
    w.capture_episode(args.frames, stage_idx)
    fb = w.bodies.fbuf
    init = fb.clone()
    stream = torch.cuda.current_stream()

    def episode():
        fb.copy_(init, non_blocking=True)
        w.run_episode(stream)

    for _ in range(max(args.warmup, 3)):
        episode()
    torch.cuda.synchronize()
    assert w.stats()["status"] == 0, "overflow during warm-up"

    def barrier():
        if world > 1:
            dist.barrier()

    # ── device-resident timed region ──
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        episode()
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ck = clocks.stop()
    ms = t0.elapsed_time(t1)
    probe = w.probe_ms()  # per-frame probed-stage durations of the last timed episode
    pairs, contacts = w.history(args.frames)
    st = w.stats()

    # ── end-to-end through the C-ABI world with host buffers ──
    host_in = init.cpu().pin_memory()
    host_out = torch.empty((13, fb.shape[1]), dtype=torch.float32).pin_memory()
    for _ in range(2):
        fb.copy_(host_in, non_blocking=True)
        w.run_episode(stream)
        host_out.copy_(fb[:13], non_blocking=True)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        fb.copy_(host_in, non_blocking=True)
        w.run_episode(stream)
        host_out.copy_(fb[:13], non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)

    if world > 1:
        ms, e2e_ms = max_over_ranks([ms, e2e_ms], device="cuda")
    body_steps = world * args.steps * args.frames * n
    value = body_steps / (ms / 1e3)
    e2e = body_steps / (e2e_ms / 1e3)

    if rank == 0:
        bytes_f = stage_bytes(args.probe_stage, n, pairs, contacts)
        achieved = float(bytes_f.sum() / (probe.sum() / 1e3) / 1e9) if probe.sum() > 0 else None
        peak, peak_kind = peaks()
        traffic = committed_traffic(args.probe_stage, float(bytes_f.mean())) if len(bytes_f) else None
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "bodies": n, "frames_per_step": args.frames,
                       "start_frame": args.start_frame,
                       "solver_mode": args.mode, "parallelism": f"replicas{world}",
                       "l2": "no flush: each step re-simulates the whole episode from its initial state, and "
                             "a frame's data (~50-130 MB touched per frame at 65k bodies, about the 126 MB L2) "
                             "is produced on the device by the previous stage or frame",
                       "mean_pairs_per_frame": float(pairs.mean()) if len(pairs) else None,
                       "mean_contacts_per_frame": float(contacts.mean()) if len(contacts) else None,
                       "contacts_per_s": float(contacts.sum() * world * args.steps / (ms / 1e3))
                       if len(contacts) else None},
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": int(host_in.numel() * 4),
                    "d2h_bytes_per_step": int(host_out.numel() * 4)},
            "roofline": {"bound": "hbm", "kernel": f"{args.probe_stage} stage (CUDA events per frame, last "
                                                    f"timed step, {len(probe)} launches)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "peak_source": f"{peak_kind} hbm_gbs", "traffic": traffic,
                         "stage_ms_per_frame": float(probe.mean()),
                         "stage_share_of_step": float(probe.sum() / (ms / args.steps))},
            "gpu_launches": int(args.steps * args.frames * kernels_per_frame(n, scene.n_scenes)),
            "clocks": ck, "overflow_status": st["status"],
        }
        if args.workload == "batch":
            line["config"]["workload"] = (f"batched forward: {scene.n_scenes} independent scenes (box stacks or "
                                          f"sphere piles, 8-256 bodies log-uniform, each on its own ground), "
                                          f"{args.frames} frames at 60 Hz, fp32, one world")
            line["config"]["scenes"] = scene.n_scenes
            line["per_scene"] = per_scene_baseline(scene, args.frames, mode, torch, device)
            line["per_scene"]["batched_over_per_scene"] = value / line["per_scene"]["value"]
        elif not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(args.bodies, args.cpu_frames)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def per_scene_baseline(scene, frames: int, mode: int, torch, device, sample: int = 64) -> dict:
    """The plain per-scene GPU path on a sample of the batch: each scene its own
    world, its frames replayed as one captured episode, scenes one after another."""
    idx = np.linspace(0, scene.n_scenes - 1, min(sample, scene.n_scenes)).astype(int)
    worlds = []
    for i in idx:
        w = device.World(scene.scene(int(i)), mode=mode)
        w.capture_episode(frames, -1)
        worlds.append((w, w.bodies.fbuf.clone()))
    stream = torch.cuda.current_stream()
    for w, init in worlds:  # warm-up
        w.bodies.fbuf.copy_(init)
        w.run_episode(stream)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for w, init in worlds:
        w.bodies.fbuf.copy_(init, non_blocking=True)
        w.run_episode(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    bodies = sum(w.scene.n_bodies for w, _ in worlds)
    return {"value": bodies * frames / (t0.elapsed_time(t1) / 1e3), "unit": METRIC,
            "sample": f"{len(worlds)} of the batch's scenes, each stepped alone ({frames} frames)"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    from oracle import oracle
    which = "ref" if oracle.ref_available() else "oracle"
    cores = os.cpu_count() or 1
    frames = max(1, args.cpu_frames // 4)
    vals = []
    for _ in range(max(args.warmup, 3) + args.steps):
        r = cpu_baseline(args.bodies, frames)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU build failed to run"}))
            return
        vals.append(r["value"])
    vals = vals[max(args.warmup, 3):]
    value = statistics.mean(vals)
    ms_step = (args.bodies + 1) * frames / value * 1e3 if value else None  # one sample of `frames` frames
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "bodies": args.bodies + 1, "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores if which == "ref" else 1,
                             "kind": "reference" if which == "ref" else "port",
                             "sample": f"frames 0-{frames - 1} of the episode per step"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.frames is None:
        args.frames = 240 if args.workload == "batch" else 600
    if args.cpu_worker:
        cpu_worker(args.cpu_worker, args.bodies, args.cpu_frames)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    run_b200(args)


if __name__ == "__main__":
    main()
