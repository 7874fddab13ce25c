"""On-disk formats of the reference's example programs, so their consumers
(the trajectory viewer, render scripts, CI golden checks) read this library's
output unchanged.

  <prefix>.scene         examples/common/scene_io.hpp:24-54  (binary)
  <prefix>.trajectory    examples/stress_test_blocks/main.cpp:172-197,
                         examples/common/scene_io.hpp:118-129 (binary)
  <prefix>.golden        examples/stress_test_blocks/main.cpp:301-316 (text)
  <prefix>.metrics.json  examples/stress_test_blocks/main.cpp:318-336 (text)

All binary files are little-endian, as the reference writes them on x86.
"""
from __future__ import annotations

import json
import struct

import numpy as np


# ── .scene: n_bodies, n_shapes (u32), body_shape_idx[n_bodies] (u32), then per
#    shape 20 bytes: u32 type, f32 half_x, half_y, half_z, u32 pad ──────────

def write_scene(prefix: str, body_shape_idx, shape_type, shape_half) -> None:
    idx = np.ascontiguousarray(body_shape_idx, np.uint32)
    st = np.asarray(shape_type, np.uint32)
    sh = np.asarray(shape_half, np.float32).reshape(-1, 3)
    if st.shape[0] != sh.shape[0]:
        raise ValueError("shape_type and shape_half differ in length")
    rec = np.zeros(st.shape[0], dtype=[("type", "<u4"), ("h", "<f4", 3), ("pad", "<u4")])
    rec["type"] = st
    rec["h"] = sh
    with open(prefix + ".scene", "wb") as f:
        f.write(struct.pack("<II", idx.shape[0], st.shape[0]))
        f.write(idx.astype("<u4").tobytes())
        f.write(rec.tobytes())


def read_scene(prefix: str):
    """(body_shape_idx [n] u32, shape_type [m] u32, shape_half [m, 3] f32)."""
    with open(prefix + ".scene", "rb") as f:
        n, m = struct.unpack("<II", f.read(8))
        idx = np.frombuffer(f.read(4 * n), "<u4").astype(np.uint32)
        rec = np.frombuffer(f.read(20 * m), dtype=[("type", "<u4"), ("h", "<f4", 3), ("pad", "<u4")])
    return idx, rec["type"].astype(np.uint32), rec["h"].astype(np.float32)


def write_scene_set(prefix: str, scene) -> None:
    """The .scene of a SceneSet (its shape catalogue as the shape table)."""
    write_scene(prefix, scene.shape, scene.shape_type, scene.shape_half)


# ── .trajectory: u32 n_bodies, u32 n_frames (simulation frames), then one
#    record per even frame: n_bodies rows of x, y, z, w, qx, qy, qz (f32) ───

def trajectory_records(n_frames: int) -> int:
    """Records in a trajectory of n_frames simulation frames (every other frame, from frame 0)."""
    return (n_frames + 1) // 2


class TrajectoryWriter:
    """Streams records into <prefix>.trajectory."""

    def __init__(self, prefix: str, n_bodies: int, n_frames: int):
        self.n_bodies = n_bodies
        self.f = open(prefix + ".trajectory", "wb")
        self.f.write(struct.pack("<II", n_bodies, n_frames))

    def write(self, records) -> None:
        r = np.ascontiguousarray(records, np.float32)
        if r.shape[-2:] != (self.n_bodies, 7):
            raise ValueError(f"records must be (..., {self.n_bodies}, 7)")
        self.f.write(r.astype("<f4").tobytes())

    def close(self) -> None:
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def write_trajectory(prefix: str, n_frames: int, records) -> None:
    r = np.asarray(records, np.float32)
    with TrajectoryWriter(prefix, r.shape[1], n_frames) as w:
        w.write(r)


def read_trajectory(prefix: str):
    """(n_bodies, n_frames, records [R, n_bodies, 7] f32)."""
    with open(prefix + ".trajectory", "rb") as f:
        n, frames = struct.unpack("<II", f.read(8))
        data = np.frombuffer(f.read(), "<f4")
    if data.size % (7 * n):
        raise ValueError("truncated trajectory")
    return n, frames, data.reshape(-1, n, 7).astype(np.float32)


# ── .golden: the final-state FNV-1a-64 as 16 lower-case hex digits + newline ─

def write_golden(prefix: str, state_hash: int) -> None:
    with open(prefix + ".golden", "w") as f:
        f.write(f"{state_hash & 0xFFFFFFFFFFFFFFFF:016x}\n")


def read_golden(prefix: str) -> int:
    with open(prefix + ".golden") as f:
        return int(f.read().strip(), 16)


# ── .metrics.json, with the reference's keys, order and number formats ──────

def write_metrics(prefix: str, n_bodies: int, n_frames: int, dt: float, wall_seconds: float,
                  avg_contacts: float) -> None:
    fps = n_frames / wall_seconds if wall_seconds > 0 else 0.0
    text = ("{\n"
            f'  "n_bodies": {n_bodies},\n'
            f'  "n_frames": {n_frames},\n'
            f'  "simulation_seconds": {n_frames * float(np.float64(np.float32(dt))):.4f},\n'
            f'  "wall_clock_seconds": {wall_seconds:.4f},\n'
            f'  "frames_per_second": {fps:.2f},\n'
            f'  "avg_contacts_per_frame": {avg_contacts:.1f},\n'
            f'  "realtime_factor": {fps / 60.0:.3f}\n'
            "}\n")
    with open(prefix + ".metrics.json", "w") as f:
        f.write(text)


def read_metrics(prefix: str) -> dict:
    with open(prefix + ".metrics.json") as f:
        return json.load(f)
