#!/usr/bin/env python3
"""Frame-step benchmark (body-steps/s) on B200.

Default workload — the batched forward configuration the headline metric
("batched vs per-scene at <= 1e-3 m drift") is quoted on: 4096 independent
scenes (box stacks or sphere piles, 8-256 bodies log-uniform, seed 3, each on
its own ground) stepped together as one world, 240 frames at 60 Hz, fp32,
synthetic seeded input. One step = one 240-frame episode of the whole batch
from its initial state, replayed as one CUDA graph.

  value       device-resident body-steps/s of the batch in sequential order
              (every scene bit-identical to the reference's sequential
              order: pose drift 0)
  per_scene   the plain per-scene GPU path (each scene its own world) on a
              sample of the same scenes, and the batched / per-scene ratio
  colored     the batch in the Jones-Plassmann coloured order: its
              body-steps/s and its pose drift and penetration against the
              sequential order
  e2e         the same metric through the C-ABI world with host buffers:
              every step uploads the initial state from pinned host memory,
              downloads the poses every other frame (the reference loop's
              trajectory, examples/stress_test_blocks/main.cpp:275-278) and
              reads the final state back
  single_scene  the large single-scene stress (65,536 bodies, 600 frames) on
              the same terms, with its own CPU baseline

`--workload single` prints the single-scene line alone.
Multi-GPU (torchrun): replicas only — each rank runs its own copy of the
workload (its own seed), no collective on the data path; the timed region is
the max over ranks. `--impl reference` times the reference's own frame-step
sources (built on the host with the SYCL shim, oracle/_ref) on the host cores
on the same workload; that arm never loads the GPU library.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "body-steps/s"
BATCH = dict(n_scenes=4096, lo=8, hi=256, seed=3, frames=240)
SINGLE = dict(bodies=65536, seed=2, frames=600)
BATCH_WORKLOAD = ("batched forward: 4096 independent scenes (jittered box stacks or sphere piles, 8-256 bodies "
                  "log-uniform, h = r = 0.4 m, each on its own ground), 240 frames at 60 Hz, fp32, one world")
SINGLE_WORKLOAD = ("large single-scene stress: 65536 bodies (70% boxes half-extent U[0.1,0.5] m, 30% spheres "
                   "r U[0.1,0.4] m, 500 kg/m^3, random rotations, v N(0,0.5) m/s) in a 40 m cube over an "
                   "80x1x80 m ground, 600 frames at 60 Hz, fp32")
STAGES = ("integrate", "broadphase", "narrowphase", "solver", "flow_solve_kernel")
MODES = {"reference": 0, "sequential": 1, "colored": 2}
FLOW_THREADS = 148 * 2 * 256  # resident threads of the dataflow solver kernel (2 blocks x 256 per SM)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="batch", choices=["batch", "single"])
    ap.add_argument("--mode", default=None, choices=list(MODES),
                    help="solver order (default: sequential for the batch, reference for the single scene)")
    ap.add_argument("--frames", type=int, default=None)
    ap.add_argument("--no-single", action="store_true", help="batch line without the single-scene object")
    ap.add_argument("--no-adjoint", action="store_true", help="batch line without the fwd+bwd objects")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-single-worker", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


_T0 = time.perf_counter()


def note(msg: str) -> None:
    """Progress of the run on stderr (wall seconds since start)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ── CPU side: the reference's own sources (oracle/_ref) on the host cores ────

def checker_kind():
    from oracle import oracle
    return "ref" if oracle.ref_available() else "oracle"


_POOL_STATE = {}


def _batch_worker_init(which: str, cfg: dict) -> None:
    from dyphur_b200 import scenes
    from oracle import oracle
    _POOL_STATE["which"] = which
    _POOL_STATE["batch"] = scenes.batch(cfg["n_scenes"], cfg["lo"], cfg["hi"], cfg["seed"],
                                        builder=oracle.scene_builder(which))


def _batch_worker_scene(job):
    """Step one scene of the batch alone on one host thread in the given solver
    order (1: XpbdSolver::set_force_serial(true)); returns (body-steps, seconds, rc)."""
    from oracle import oracle
    i, frames, mode = job
    sc = _POOL_STATE["batch"].scene(i)
    w = oracle.World(sc, _POOL_STATE["which"])
    t0 = time.perf_counter()
    rc = w.step(frames, mode)
    dt = time.perf_counter() - t0
    w.close()
    return sc.n_bodies * frames, dt, rc


class BatchCpu:
    """The reference build stepping scenes of the batch one per host core (the
    reference steps one scene at a time; independent scenes run side by side)."""

    def __init__(self, cfg: dict, cores: int):
        self.which = checker_kind()
        self.cfg = cfg
        self.cores = cores
        env_omp = os.environ.get("OMP_NUM_THREADS")
        os.environ["OMP_NUM_THREADS"] = "1"  # one thread per scene; inherited by the spawned workers
        ctx = mp.get_context("spawn")
        self.pool = ctx.Pool(cores, initializer=_batch_worker_init, initargs=(self.which, cfg))
        if env_omp is None:
            del os.environ["OMP_NUM_THREADS"]
        else:
            os.environ["OMP_NUM_THREADS"] = env_omp

    def run(self, scene_ids, frames: int, mode: int = 1):
        """Whole-job wall time of stepping these scenes on all workers."""
        t0 = time.perf_counter()
        res = self.pool.map(_batch_worker_scene, [(int(i), frames, mode) for i in scene_ids], chunksize=1)
        wall = time.perf_counter() - t0
        if any(r[2] != 0 for r in res):
            raise RuntimeError("reference build returned an error")
        return sum(r[0] for r in res), wall, sum(r[1] for r in res)

    def close(self):
        self.pool.close()
        self.pool.join()


def batch_cpu_baseline(cfg: dict, sample_stride: int = 4) -> dict | None:
    cores = os.cpu_count() or 1
    try:
        cpu = BatchCpu(cfg, cores)
        ids = np.arange(0, cfg["n_scenes"], sample_stride)
        bs, wall, _ = cpu.run(ids, cfg["frames"])
        one = np.arange(0, cfg["n_scenes"], cfg["n_scenes"] // 16)
        bs1, _, busy1 = cpu.run(one, cfg["frames"])
        cpu.close()
    except Exception as e:  # the baseline is reported, not required
        print(f"cpu baseline failed: {e}", file=sys.stderr)
        return None
    kind = "reference" if cpu.which == "ref" else "port"
    return {"value": bs / wall, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"every {sample_stride}th scene of the batch ({len(ids)} scenes, {cfg['frames']} frames each, "
                      f"{wall:.1f} s), one scene per host core, sequential order (set_force_serial)",
            "single_thread": {"value": bs1 / busy1, "unit": METRIC, "cores": 1,
                              "sample": f"{len(one)} scenes, {cfg['frames']} frames each, per-scene step time"}}


def _single_cpu_worker(spec: str) -> None:
    """Child process: the reference build on the pile. spec = 'full:<frames>'
    times frames 0..frames-1; 'windows:<w>:<n>:<total>' steps the episode
    untimed saving checkpoints every w frames, then times n windows of w
    frames each, cycling over the episode from its checkpoints;
    'ckpt:<file.npy>:<w>' times a window of w frames from each state in the
    file (states the GPU path produced; it is bit-identical to the reference at
    every frame of this episode, tests/test_gpu_late_frames.py)."""
    from dyphur_b200 import scenes
    from oracle import oracle
    which = checker_kind()
    s = scenes.random_pile(SINGLE["bodies"], SINGLE["seed"], builder=oracle.scene_builder(which))
    w = oracle.World(s, which)
    parts = spec.split(":")
    out = {"bodies": s.n_bodies, "which": which}
    if parts[0] == "full":
        frames = int(parts[1])
        t0 = time.perf_counter()
        rc = w.step(frames, 0)
        out.update(rc=rc, seconds=time.perf_counter() - t0, frames=frames)
        print(json.dumps(out), flush=True)
        return
    if parts[0] == "ckpt":
        ckpt = list(np.load(parts[1]))
        win, n_win = int(parts[2]), len(ckpt)
    else:
        win, n_win, total = int(parts[1]), int(parts[2]), int(parts[3])
        ckpt = []
        for f in range(0, total, win):
            ckpt.append(w.state())
            w.step(win, 0)
    secs = []
    for k in range(n_win):
        w.set_state(ckpt[k % len(ckpt)])
        t0 = time.perf_counter()
        rc = w.step(win, 0)
        secs.append(time.perf_counter() - t0)
        if rc != 0:
            out["rc"] = rc
            break
    out.update(rc=out.get("rc", 0), window_seconds=secs, frames=win)
    print(json.dumps(out), flush=True)


def run_single_cpu(spec: str, threads: int, timeout: int = 1200) -> dict:
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-single-worker", spec]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=timeout, check=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def single_cpu_baseline(frames: int, ckpt_states: np.ndarray, ckpt_frames, win: int) -> dict | None:
    """The reference build on windows of `win` frames spread over the episode,
    each started from the GPU path's state at that frame, OpenMP on every core;
    plus frames 0-9 on one thread."""
    import tempfile
    cores = os.cpu_count() or 1
    try:
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "ckpt.npy")
            np.save(path, ckpt_states)
            r = run_single_cpu(f"ckpt:{path}:{win}", cores)
        r1 = run_single_cpu("full:10", 1)
    except Exception as e:
        print(f"cpu baseline failed: {e}", file=sys.stderr)
        return None
    if r["rc"] != 0 or r1["rc"] != 0:
        return None
    kind = "reference" if r["which"] == "ref" else "port"
    secs = sum(r["window_seconds"])
    return {"value": r["bodies"] * win * len(r["window_seconds"]) / secs, "unit": METRIC, "cores": cores,
            "kind": kind,
            "sample": f"{len(ckpt_frames)} windows of {win} frames starting at frames {list(ckpt_frames)} of the "
                      f"{frames}-frame episode ({secs:.1f} s), each from the state the GPU path reached there, "
                      f"OpenMP on every core",
            "single_thread": {"value": r1["bodies"] * 10 / r1["seconds"], "unit": METRIC, "cores": 1,
                              "sample": "frames 0-9 of the episode, one thread"}}


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


# ── algorithmic bytes ────────────────────────────────────────────────────────

def frame_bytes(n: int, pairs: np.ndarray, contacts: np.ndarray) -> np.ndarray:
    """Compulsory bytes of one frame (each input read once, each output written
    once): 424 per body, 32 per candidate pair, 72 per contact."""
    return 424.0 * n + 32.0 * pairs.astype(np.float64) + 72.0 * contacts.astype(np.float64)


def flow_kernel_bytes(n: int, contacts: np.ndarray) -> np.ndarray:
    """Compulsory bytes of one dataflow-solver launch: per body the state it
    reads (80 B: pose, velocities, inverse mass and inertia) and writes (52 B),
    per contact its 36-byte row."""
    return 132.0 * n + 36.0 * contacts.astype(np.float64)


def frame_kernel_bytes(n: int, pairs: np.ndarray, contacts: np.ndarray) -> np.ndarray:
    """Compulsory bytes of one fused batched-frame launch (scene_frame_kernel):
    per body the state it reads (80 B), its shape index, flags, shape type and
    half extents (24 B) and the state it writes (52 B); per stored pair its
    4-byte record; per contact its 36-byte row and 4-byte colour. Pairs and
    contacts otherwise live in shared memory."""
    return 156.0 * n + 4.0 * pairs.astype(np.float64) + 40.0 * contacts.astype(np.float64)


def flow_kernel_active(contacts: np.ndarray, mode: int) -> np.ndarray:
    """Frames on which the dataflow kernel does the solve: the sequential order
    at <= 2048 contacts and the reference order at <= 256 run the one-block
    kernel, empty frames nothing, more than 16 contacts per resident thread the
    round-synchronous kernel."""
    c = contacts.astype(np.int64)
    seq = (mode == 1) | ((mode == 0) & (c <= 256))
    return (c > 0) & ~(seq & (c <= 2048)) & (c <= 16 * FLOW_THREADS)


def kernels_per_frame(n: int, n_scenes: int = 1, fused: bool = False) -> int:
    """Library kernels one frame launches (matches the ncu launch lists in profiles/)."""
    if fused:  # the fused frame kernel and the frame's statistics
        return 2
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


def committed_traffic(key: str, mean_algorithmic_bytes: float):
    """DRAM bytes per launch of the kernel from the committed ncu capture
    (profiles/traffic.json), scaled from the captured launch's units to the
    mean launch by the ratio of algorithmic bytes."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            rec = json.load(f)[key]
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


# ── GPU side ─────────────────────────────────────────────────────────────────

def timed_episodes(w, steps, warmup, torch, barrier, clocks=None):
    """Device time (ms) of `steps` episodes, each from the world's initial state."""
    fb = w.bodies.fbuf
    init = fb.clone()
    stream = torch.cuda.current_stream()

    def episode():
        fb.copy_(init, non_blocking=True)
        w.run_episode(stream)

    for _ in range(max(warmup, 3)):
        episode()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        episode()
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ck = clocks.stop() if clocks else None
    fb.copy_(init)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1), ck, init


def e2e_episodes(w, init, frames, steps, torch, barrier):
    """The same episodes through the C-ABI world with host buffers: initial
    state uploaded from pinned memory, poses downloaded every other frame into
    a pinned trajectory buffer, final state read back."""
    fb = w.bodies.fbuf
    n = w.bodies.n
    stream = torch.cuda.current_stream()
    host_in = init.cpu().pin_memory()
    host_out = torch.empty((13, fb.shape[1]), dtype=torch.float32).pin_memory()
    records = (frames + 1) // 2
    traj = torch.empty((records, n, 7), dtype=torch.float32).pin_memory()
    w.set_trajectory(traj, 2)
    w.capture_episode(frames, -1)

    def step():
        fb.copy_(host_in, non_blocking=True)
        w.run_episode(stream)
        host_out.copy_(fb[:13], non_blocking=True)

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    w.set_trajectory(None)
    h2d = host_in.numel() * 4
    d2h = host_out.numel() * 4 + traj.numel() * 4
    return ms, h2d, d2h


def probe_flow_kernel(w, frames, mode, torch, fused=False):
    """Per-frame device time of the dominant kernel alone (events in the
    episode graph around that launch), the counts of the frames, and the
    roofline of that kernel: the dataflow solver kernel of a single scene, or
    the fused frame kernel of a batch whose frames run fused."""
    stream = torch.cuda.current_stream()
    fb = w.bodies.fbuf
    init = fb.clone()
    w.capture_episode(frames, STAGES.index("flow_solve_kernel"))
    for _ in range(2):
        fb.copy_(init)
        w.run_episode(stream)
    torch.cuda.synchronize()
    probe = w.probe_ms()
    pairs, contacts = w.history(frames)
    fb.copy_(init)
    torch.cuda.synchronize()
    n = w.bodies.n
    if fused:
        kernel = "scene_frame_kernel"
        act = np.ones(frames, bool)
        b = frame_kernel_bytes(n, pairs, contacts)
        rule = ("156 B per body (read state 80 + shape and flags 24, write state 52) + 4 B per stored pair + "
                "40 B per contact (row 36 + colour 4)")
    else:
        kernel = "flow_solve_kernel"
        act = flow_kernel_active(contacts, mode)
        b = flow_kernel_bytes(n, contacts)
        rule = "132 B per body (read 80, write 52) + 36 B per contact row"
    peak, peak_kind = peaks()
    achieved = float(b[act].sum() / (probe[act].sum() / 1e3) / 1e9) if act.any() and probe[act].sum() > 0 else None
    out = {"bound": "hbm", "kernel": kernel, "launches_timed": int(act.sum()),
           "algorithmic_bytes_per_launch": float(b[act].mean()) if act.any() else None,
           "bytes_rule": rule, "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": (achieved / peak) if achieved else None, "peak_source": f"{peak_kind} hbm_gbs",
           "traffic": committed_traffic(kernel, float(b[act].mean())) if act.any() else None,
           "kernel_ms_per_launch": float(probe[act].mean()) if act.any() else None}
    if fused and act.any():  # the frame's compulsory bytes over the one launch that does the whole frame
        fb_ = frame_bytes(n, pairs, contacts)
        out["frame_rule_achieved"] = float(fb_.sum() / (probe.sum() / 1e3) / 1e9)
        out["frame_rule_frac"] = out["frame_rule_achieved"] / peak
    return out, pairs, contacts, probe


def gpu_workload(scene, mode, frames, args, torch, barrier, clocks=None, roofline=True):
    from dyphur_b200 import device
    w = device.World(scene, mode=mode)
    tuned = None
    if scene.n_scenes > 1:  # tuned on the episode's first half from its initial state, before it is captured
        tuned = w.autotune(max(16, frames // 2))
        torch.cuda.synchronize()
    w.capture_episode(frames, -1)
    ms, ck, init = timed_episodes(w, args.steps, args.warmup, torch, barrier, clocks)
    st = w.stats()
    out = {"ms": ms, "clocks": ck, "status": st["status"], "world": w, "init": init, "fused_config": tuned}
    if roofline:
        out["roofline"], out["pairs"], out["contacts"], _ = probe_flow_kernel(w, frames, mode, torch,
                                                                              fused=scene.n_scenes > 1)
    return out


def fp64_error_report(scene, mode: int, frames: int, sample: int = 8, carried=(10, 30)) -> dict:
    """Error of the float frame step against an FP64 re-run of the same
    frames along the float run's contact set and branches
    (oracle/dual_oracle.cpp, dyd_fp64_run), on a sample of the scenes, in
    solver order `mode`. The per-frame figure restarts the FP64 run from the
    float state every frame (each frame's own rounding error); the carried
    figure keeps the FP64 state, which contact-rich scenes amplify like any
    perturbation, so it is given only over the first frames."""
    from dyphur_b200 import device
    from oracle import oracle
    idx = np.linspace(0, scene.n_scenes - 1, min(sample, scene.n_scenes)).astype(int)
    per_frame_max, per_frame_mean, rot_max, carried_max = [], [], [], {c: 0.0 for c in carried}
    for i in idx:
        sc = scene.scene(int(i)) if scene.n_scenes > 1 else scene
        st, im, ii, fl = device.pack_bodies(sc)
        args = (st, im, ii, sc.shape_type[sc.shape], np.ascontiguousarray(sc.shape_half[sc.shape].T), fl)
        ep, er, _, _ = oracle.fp64_run(*args, frames, sc.dt, sc.gravity, sc.n_substeps, sc.n_iters, sc.friction,
                                       mode, local=True)
        per_frame_max.append(float(ep.max()))
        per_frame_mean.append(float(ep.mean()))
        rot_max.append(float(er.max()))
        epc, _, _, _ = oracle.fp64_run(*args, max(carried), sc.dt, sc.gravity, sc.n_substeps, sc.n_iters,
                                       sc.friction, mode, local=False)
        for c in carried:
            carried_max[c] = max(carried_max[c], float(epc[c - 1]))
    return {"vs": "FP64 re-run of the same frames along the float run's contacts and branches",
            "solver_mode": {0: "reference", 1: "sequential", 2: "colored"}[mode],
            "sample": f"{len(idx)} scenes, {frames} frames" if scene.n_scenes > 1 else f"{frames} frames",
            "per_frame_pos_err_max_m": max(per_frame_max), "per_frame_pos_err_mean_m": float(np.mean(per_frame_mean)),
            "per_frame_rot_err_max": max(rot_max),
            "carried_pos_err_max_m": {str(c): carried_max[c] for c in carried}}


def final_state(scene, mode, frames, torch):
    from dyphur_b200 import device
    w = device.World(scene, mode=mode)
    w.step(frames)
    torch.cuda.synchronize()
    st = w.state()
    _, p7 = w.contacts()
    w.close()
    return st, p7


def drift_report(scene, frames, torch) -> dict:
    """Coloured order against the sequential order on the batch: pose drift
    (max over bodies of the position distance, and of the rotation angle) at
    a few frames and after the episode, the one-frame drift from a shared
    state, and the penetration (contact depth) after the last frame."""
    from dyphur_b200 import device
    ws, wc = device.World(scene, mode=1), device.World(scene, mode=2)
    at, out, cur = (10, 30, 60, 120, frames), {}, 0
    for f in at:
        ws.step(f - cur)
        wc.step(f - cur)
        cur = f
        a, b = ws.state(), wc.state()
        dp = np.sqrt(((a[:3] - b[:3]) ** 2).sum(0))
        dq = np.abs((a[3:7] * b[3:7]).sum(0)).clip(0.0, 1.0)
        out[f] = (float(dp.max()), float(2.0 * np.arccos(dq).max()))
    one = []
    sq = device.World(scene, mode=1)
    cur = 0
    for f in (30, 120, frames - 2):
        sq.step(f - cur)
        wc.bodies.set_state(sq.state())
        sq.step(1)
        wc.step(1)
        cur = f + 1
        one.append(float(np.sqrt(((sq.state()[:3] - wc.state()[:3]) ** 2).sum(0)).max()))
    _, cs = ws.contacts()
    _, cc = wc.contacts()
    for x in (ws, wc, sq):
        x.close()
    return {"vs": "sequential order, same scenes, same initial state",
            "max_pose_drift_m": out[frames][0], "max_rot_drift_rad": out[frames][1],
            "max_pose_drift_m_at_frame": {str(f): out[f][0] for f in at},
            "one_frame_drift_m": one, "one_frame_drift_frames": [30, 120, frames - 2],
            "penetration_after_settling_m": {"colored_max": float(cc[:, 6].max()) if len(cc) else 0.0,
                                             "colored_mean": float(cc[:, 6].mean()) if len(cc) else 0.0,
                                             "sequential_max": float(cs[:, 6].max()) if len(cs) else 0.0,
                                             "sequential_mean": float(cs[:, 6].mean()) if len(cs) else 0.0},
            "within_1e-3_m": out[frames][0] <= 1e-3}


def _dual_error(w, scene, i, frames, g_vel, g_ang, g_im, at_float, loss_mask, scale, max_params=90):
    """Relative error of the adjoint's gradient for scene i of a batch against
    the FP64 dual-number oracle (oracle/dual_oracle.cpp) over the same frames;
    the batch loss is `scale` times the sum of the scenes' masked losses."""
    from oracle import oracle
    b0, b1 = int(scene.body_offset[i]), int(scene.body_offset[i + 1])
    fb = w.bodies.fbuf.cpu().numpy()
    n = b1 - b0
    im = fb[13, b0:b1].copy()
    dyn = [j for j in range(n) if im[j] != 0]
    params = [(k, dyn[-1]) for k in range(6)] + [(6, j) for j in dyn][:max_params - 6]
    mask = loss_mask[b0:b1].astype(np.uint8)
    tg = scene.targets[b0:b1]
    _, g_d, _, _ = oracle.dual_rollout(np.ascontiguousarray(w.initial[:, b0:b1].cpu().numpy()), im,
                                       np.ascontiguousarray(fb[14:20, b0:b1]), scene.shape_type[scene.shape[b0:b1]],
                                       np.ascontiguousarray(scene.shape_half[scene.shape[b0:b1]].T),
                                       scene.flags[b0:b1], frames, scene.dt, scene.gravity, scene.n_substeps,
                                       scene.n_iters, scene.friction, params, tg, mask, at_float=at_float)
    g = []
    for k, j in params:
        g.append(g_vel[b0 + j, k] if k < 3 else (g_ang[b0 + j, k - 3] if k < 6 else g_im[b0 + j]))
    g = np.array(g, np.float64) / scale
    return float(np.linalg.norm(g - g_d) / max(np.linalg.norm(g_d), 1e-30))


def adjoint_report(torch, scene, frames: int, every: int, label: str, loss_mask, reps: int = 3,
                   checker: bool = True) -> dict:
    """Forward rollout and forward + adjoint of a differentiable batch
    (sequential order), loss = mean over the masked bodies of |x_final -
    target|^2: body-steps/s of each, their ratio, the device memory the
    adjoint keeps, and the gradient error against the FP64 oracle."""
    from dyphur_b200 import device
    from dyphur_b200.autograd import rollout
    w = device.World(scene, mode=1)
    tuned = w.autotune(frames)  # the fused frame's configuration (no frame changes); records use it too
    n = scene.n_bodies
    stream = torch.cuda.current_stream()
    dyn = torch.from_numpy(loss_mask.astype(np.float32)).cuda()
    scale = 1.0 / float(loss_mask.sum())
    tgt = torch.from_numpy(scene.targets).cuda()

    def once(fr):
        vel = w.initial[7:10, :n].T.clone().requires_grad_(True)
        ang = w.initial[10:13, :n].T.clone().requires_grad_(True)
        im = w.bodies.fbuf[13, :n].clone().requires_grad_(True)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        fin = rollout(w, vel, ang, im, fr, every=min(every, fr))
        e[1].record(stream)
        pos = fin[:3].T
        loss = (((pos - tgt) ** 2).sum(1) * dyn).sum() * scale
        loss.backward()
        e[2].record(stream)
        torch.cuda.synchronize()
        return e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), vel.grad, ang.grad, im.grad

    once(frames)  # warm-up
    tf, tb = [], []
    for _ in range(reps):
        a, b, gv, ga, gm = once(frames)
        tf.append(a)
        tb.append(b)
    fwd_ms, bwd_ms = statistics.median(tf), statistics.median(tb)
    gv, ga, gm = gv.cpu().numpy(), ga.cpu().numpy(), gm.cpu().numpy()
    per_frame = None
    if every > 1:  # the same with a checkpoint at every frame (no segment recompute)
        every_cfg = every
        every = 1
        a, b, _, _, _ = once(frames)
        a, b, _, _, _ = once(frames)
        per_frame = (a + b) / a
        every = every_cfg
    err_full = err_10 = None
    if checker:  # the CPU checker leg: FP64 dual numbers (oracle/) on scene 0
        err_full = _dual_error(w, scene, 0, frames, gv, ga, gm, True, loss_mask, scale)
        _, _, gv10, ga10, gm10 = once(10)
        err_10 = _dual_error(w, scene, 0, 10, gv10.cpu().numpy(), ga10.cpu().numpy(), gm10.cpu().numpy(), False,
                             loss_mask, scale)
    # checkpoints, the states of two segments, one record set per frame of two
    # segments (36 record and 13 word rows per contact slot, 11 rows per
    # body), the two adjoint states
    n_ckpt = (frames + every - 1) // every
    slots = int(sum(max(64, 16 * int(b) + 64) for b in np.diff(scene.body_offset)))
    set_bytes = 4 * ((36 + 13) * slots + 11 * n)
    group = every if every > 1 else max(1, min(4, (2 << 30) // (2 * set_bytes)))
    seg = min(group, frames)
    states = 2 * (seg - 1) * 13 * n if every > 1 else 0
    act = 4 * (n_ckpt * 13 * n + states + 2 * 13 * n) + 2 * seg * set_bytes
    reverse = w.adjoint_config()
    w.close()
    return {"workload": label, "scenes": scene.n_scenes, "bodies": n, "frames": frames,
            "checkpoint_every": every, "solver_mode": "sequential", "fused_config": tuned,
            "reverse_config": reverse,
            "fwd": {"value": n * frames / (fwd_ms / 1e3), "unit": METRIC, "ms": fwd_ms},
            "fwd_bwd": {"value": n * frames / ((fwd_ms + bwd_ms) / 1e3), "unit": METRIC, "ms": fwd_ms + bwd_ms},
            "fwd_bwd_over_fwd": (fwd_ms + bwd_ms) / fwd_ms,
            "fwd_bwd_over_fwd_checkpoint_every_frame": per_frame,
            "adjoint_device_bytes": act,
            "grad_rel_err_vs_fp64": {"scene": 0, "frames_10_fp64_values": err_10,
                                     f"frames_{frames}_fp64_at_float_values": err_full},
            "grads": "initial velocities and spins, inverse masses (inverse inertia held fixed)"}


def per_scene_baseline(scene, frames: int, mode: int, torch, sample: int = 32) -> dict:
    """The plain per-scene GPU path on a sample of the batch: each scene its own
    world, its frames replayed as one captured episode, scenes one after another."""
    from dyphur_b200 import device
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
    for w, _ in worlds:
        w.close()
    return {"value": bodies * frames / (t0.elapsed_time(t1) / 1e3), "unit": METRIC,
            "sample": f"{len(worlds)} of the batch's scenes, each stepped alone as its own world ({frames} frames)"}


def single_line(args, torch, barrier, world, rank, local, seed, frames, mode_name, nested) -> dict:
    from dyphur_b200 import scenes
    mode = MODES[mode_name]
    scene = scenes.random_pile(SINGLE["bodies"], seed=seed)
    n = scene.n_bodies
    steps = args.steps if not nested else min(args.steps, 5)
    a = argparse.Namespace(steps=steps, warmup=args.warmup if not nested else 3)
    clocks = Clocks(local) if not nested else None
    r = gpu_workload(scene, mode, frames, a, torch, barrier, clocks)
    w = r["world"]
    e2e_ms, h2d, d2h = e2e_episodes(w, r["init"], frames, steps, torch, barrier)
    ms = r["ms"]
    if world > 1:
        ms, e2e_ms = max_over_ranks([ms, e2e_ms], device="cuda")
    body_steps = world * steps * frames * n
    pairs, contacts = r["pairs"], r["contacts"]
    fb_ = frame_bytes(n, pairs, contacts)
    peak, peak_kind = peaks()
    frame_ach = float(fb_.sum() / (ms / steps / 1e3) / 1e9)
    line = {"metric": METRIC, "value": body_steps / (ms / 1e3), "unit": METRIC, "n_gpus": world, "steps": steps,
            "warmup": a.warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": SINGLE_WORKLOAD, "bodies": n, "frames_per_step": frames, "seed": seed,
                       "solver_mode": mode_name, "parallelism": f"replicas{world}",
                       "l2": "no flush: each step re-simulates the whole episode from its initial state; a frame "
                             "touches ~50-130 MB (about the 126 MB L2), produced on the device by the frame before",
                       "mean_pairs_per_frame": float(pairs.mean()), "mean_contacts_per_frame": float(contacts.mean()),
                       "contacts_per_s": float(contacts.sum() * world * steps / (ms / 1e3))},
            "e2e": {"value": body_steps / (e2e_ms / 1e3), "unit": METRIC, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "trajectory_every_frames": 2},
            "roofline": r["roofline"],
            "frame_roofline": {"bound": "hbm", "achieved": frame_ach, "peak": peak, "unit": "GB/s",
                               "frac": frame_ach / peak, "peak_source": f"{peak_kind} hbm_gbs",
                               "bytes_rule": "424 B per body + 32 B per candidate pair + 72 B per contact, per frame"},
            "gpu_launches": int(steps * frames * kernels_per_frame(n)),
            "clocks": r["clocks"], "overflow_status": r["status"]}
    w.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from dyphur_b200 import device
        win, starts = 5, list(range(0, frames, max(1, frames // 10)))
        cw = device.World(scene, mode=mode)
        states, cur = [], 0
        for f in starts:
            cw.step(f - cur)
            cur = f
            states.append(cw.state())
        cw.close()
        note("single scene timed")
        line["cpu_baseline"] = single_cpu_baseline(frames, np.stack(states), starts, win)
    return line


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    if args.workload == "single":
        line = single_line(args, torch, barrier, world, rank, local, SINGLE["seed"] + rank, args.frames,
                           args.mode or "reference", nested=False)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    from dyphur_b200 import scenes
    frames = args.frames
    mode_name = args.mode or "sequential"
    mode = MODES[mode_name]
    scene = scenes.batch(BATCH["n_scenes"], BATCH["lo"], BATCH["hi"], seed=BATCH["seed"] + rank)
    n = scene.n_bodies
    clocks = Clocks(local)
    note("batch scene built")
    r = gpu_workload(scene, mode, frames, args, torch, barrier, clocks)
    note("batch timed + flow probe")
    w = r["world"]
    e2e_ms, h2d, d2h = e2e_episodes(w, r["init"], frames, args.steps, torch, barrier)
    w.close()
    note("batch e2e")
    # the coloured order on the same batch, for the drift / speed trade
    rc = gpu_workload(scene, MODES["colored"], frames, argparse.Namespace(steps=args.steps, warmup=3), torch,
                      barrier, None, roofline=False)
    rc["world"].close()
    note("batch coloured")
    ms, ms_c = r["ms"], rc["ms"]
    if world > 1:
        ms, e2e_ms, ms_c = max_over_ranks([ms, e2e_ms, ms_c], device="cuda")
    body_steps = world * args.steps * frames * n
    value = body_steps / (ms / 1e3)
    value_c = body_steps / (ms_c / 1e3)
    if rank == 0:
        pairs, contacts = r["pairs"], r["contacts"]
        fb_ = frame_bytes(n, pairs, contacts)
        peak, peak_kind = peaks()
        frame_ach = float(fb_.sum() / (ms / args.steps / 1e3) / 1e9)
        per_scene = per_scene_baseline(scene, frames, mode, torch)
        per_scene["batched_over_per_scene"] = value / per_scene["value"]
        note("per-scene path")
        drift = drift_report(scene, frames, torch)
        note("drift")
        stress = scenes.stress_blocks()
        config1 = {"workload": "the reference's stress_test_blocks scene: 1024 boxes (8x16x8, spacing 0.85 m, "
                               "jitter 0.01) + ground",
                   "colored_drift": drift_report(stress, 300, torch)}
        fp64 = None
        if not args.no_cpu_baseline:  # the CPU checker leg: FP64 re-runs (oracle/) beside the GPU numbers
            fp64 = [fp64_error_report(scene, mode, frames, sample=6), fp64_error_report(scene, 2, frames, sample=6)]
            config1["fp64_error"] = fp64_error_report(stress, 0, 120, sample=1)
        note("fp64 error + config-1 drift")
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD, "scenes": scene.n_scenes, "bodies": n, "frames_per_step": frames,
                       "seed": BATCH["seed"], "solver_mode": mode_name, "parallelism": f"replicas{world}",
                       "pose_drift_vs_sequential_m": 0.0 if mode == 1 else None,
                       "l2": "no flush: each step re-simulates the whole episode from its initial state; the "
                             "batch's per-frame data (bodies 26 MB, pairs and contacts ~30 MB) is produced on the "
                             "device by the frame before",
                       "mean_pairs_per_frame": float(pairs.mean()), "mean_contacts_per_frame": float(contacts.mean()),
                       "contacts_per_s": float(contacts.sum() * world * args.steps / (ms / 1e3))},
            "per_scene": per_scene,
            "colored": {"value": value_c, "unit": METRIC, "ms_per_step": ms_c / args.steps,
                        "over_per_scene": value_c / per_scene["value"], "over_sequential": value_c / value,
                        "drift": drift},
            "fp64_error": fp64,
            "config1": config1,
            "e2e": {"value": body_steps / (e2e_ms / 1e3), "unit": METRIC, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "trajectory_every_frames": 2},
            "roofline": r["roofline"],
            "frame_roofline": {"bound": "hbm", "achieved": frame_ach, "peak": peak, "unit": "GB/s",
                               "frac": frame_ach / peak, "peak_source": f"{peak_kind} hbm_gbs",
                               "bytes_rule": "424 B per body + 32 B per candidate pair + 72 B per contact, per frame"},
            "gpu_launches": int(args.steps * frames * kernels_per_frame(n, scene.n_scenes,
                                                                       fused=r["fused_config"] is not None)),
            "fused_config": r["fused_config"], "colored_fused_config": rc["fused_config"],
            "clocks": r["clocks"], "overflow_status": r["status"],
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = batch_cpu_baseline(dict(BATCH, frames=frames))
            note("batch cpu baseline")
        if not args.no_adjoint and world == 1:
            push = scenes.push(256, seed=4)
            boxes = np.zeros(push.n_bodies, bool)
            for i in range(push.n_scenes):
                boxes[push.body_offset[i]:push.body_offset[i] + 64] = True
            mixed = scenes.batch_mixed(1024, 16, 512, seed=5)
            line["adjoint"] = [
                adjoint_report(torch, push, 120, 10, checker=not args.no_cpu_baseline, label=
                               "differentiable push: 256 scenes of 64 boxes + a 5 kg pusher, loss = mean squared "
                               "distance of the boxes' final centroids to seeded targets, 120 frames", loss_mask=boxes),
                adjoint_report(torch, mixed, 60, 1, checker=not args.no_cpu_baseline, label=
                               "batched fwd+bwd: 1024 scenes of 16-512 mixed boxes / spheres, loss = mean squared "
                               "final position of every dynamic body, 60 frames", loss_mask=mixed.mass > 0)]
            note("adjoint")
        if not args.no_single and world == 1:
            line["single_scene"] = single_line(args, torch, barrier, 1, 0, local, SINGLE["seed"], SINGLE["frames"],
                                               "reference", nested=True)
            note("single scene")
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ── reference arm ────────────────────────────────────────────────────────────

def run_reference(args) -> None:
    rank, _, _ = rank_info()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    warm = max(args.warmup, 3)
    try:
        if args.workload == "batch":
            cfg = dict(BATCH, frames=args.frames)
            cpu = BatchCpu(cfg, cores)
            which = cpu.which
            # step k takes the next slice of the batch's scenes, so K steps cover the batch in order
            per = -(-cfg["n_scenes"] // max(args.steps, 1))
            ids = np.arange(cfg["n_scenes"])
            for k in range(warm):
                cpu.run(ids[(k * per) % cfg["n_scenes"]:][:max(1, per // 4)], cfg["frames"])
            bs_tot, wall_tot, walls = 0, 0.0, []
            for k in range(args.steps):
                sl = np.take(ids, np.arange(k * per, (k + 1) * per), mode="wrap")
                bs, wall, _ = cpu.run(sl, cfg["frames"])
                bs_tot += bs
                wall_tot += wall
                walls.append(wall)
            cpu.close()
            value = bs_tot / wall_tot
            config = {"workload": BATCH_WORKLOAD, "scenes": cfg["n_scenes"], "frames_per_step": cfg["frames"],
                      "seed": cfg["seed"], "solver_mode": "sequential", "parallelism": "host, one scene per core"}
            sample = (f"step k steps scenes [k*{per}, (k+1)*{per}) of the batch (wrapping), {cfg['frames']} frames "
                      f"each, one scene per host core; {args.steps} steps cover "
                      f"{min(args.steps * per, cfg['n_scenes'])} of {cfg['n_scenes']} scenes")
            ms_step = 1e3 * wall_tot / args.steps
        else:
            frames = args.frames
            win = 30
            r = run_single_cpu(f"windows:{win}:{warm + args.steps}:{frames}", cores)
            which = r["which"]
            if r["rc"] != 0:
                raise RuntimeError(f"reference build returned {r['rc']}")
            secs = r["window_seconds"][warm:]
            value = r["bodies"] * win * len(secs) / sum(secs)
            config = {"workload": SINGLE_WORKLOAD, "bodies": r["bodies"], "frames_per_step": win,
                      "seed": SINGLE["seed"], "solver_mode": "reference", "parallelism": "host OpenMP"}
            sample = (f"step k steps frames [30k, 30k+30) of the {frames}-frame episode from a checkpoint "
                      f"(wrapping); {args.steps} steps cover {min(args.steps * win, frames)} of {frames} frames")
            ms_step = 1e3 * sum(secs) / len(secs)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed to run: {e}"}))
        return
    kind = "reference" if which == "ref" else "port"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": warm, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.cpu_single_worker:
        _single_cpu_worker(args.cpu_single_worker)
        return
    if args.frames is None:
        args.frames = BATCH["frames"] if args.workload == "batch" else SINGLE["frames"]
    if args.impl == "reference":
        run_reference(args)
        return
    run_b200(args)


if __name__ == "__main__":
    main()
