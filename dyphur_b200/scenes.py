"""Synthetic scene sets (host numpy arrays) built by the library's C++ builders.

The builders live in ``csrc/scenes.cpp`` and are exported through the C ABI
(``dyph_scene_make``); this module copies a built set into numpy arrays.
Every builder takes an optional ``builder=(cdll, prefix)``: the CPU checkers
in ``oracle/`` carry the same builders as ``dyo_scene_make`` /
``dyr_scene_make``, so a CPU-only run builds identical scenes without
loading the GPU library.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._lib import load_library

BOX_GRID, DETERMINISM, RANDOM_PILE, BATCH, PUSH, BATCH_MIXED = range(6)


class _SceneSetC(ctypes.Structure):
    _fields_ = [
        ("n_scenes", ctypes.c_uint32), ("n_bodies", ctypes.c_uint32), ("n_shapes", ctypes.c_uint32),
        ("pos", ctypes.POINTER(ctypes.c_float)), ("rot", ctypes.POINTER(ctypes.c_float)),
        ("vel", ctypes.POINTER(ctypes.c_float)), ("ang", ctypes.POINTER(ctypes.c_float)),
        ("mass", ctypes.POINTER(ctypes.c_float)), ("inertia", ctypes.POINTER(ctypes.c_float)),
        ("shape", ctypes.POINTER(ctypes.c_uint32)), ("flags", ctypes.POINTER(ctypes.c_uint32)),
        ("shape_type", ctypes.POINTER(ctypes.c_uint32)), ("shape_half", ctypes.POINTER(ctypes.c_float)),
        ("body_offset", ctypes.POINTER(ctypes.c_uint32)), ("shape_offset", ctypes.POINTER(ctypes.c_uint32)),
        ("bounds", ctypes.POINTER(ctypes.c_float)), ("targets", ctypes.POINTER(ctypes.c_float)),
        ("max_pairs", ctypes.c_uint32), ("max_contacts", ctypes.c_uint32),
        ("dt", ctypes.c_float), ("n_iters", ctypes.c_int32), ("friction", ctypes.c_float),
    ]


@dataclass
class SceneSet:
    """Host description of one or more independent scenes (BodyParams fields)."""

    pos: np.ndarray          # (n, 3) float32
    rot: np.ndarray          # (n, 4) float32, w x y z
    vel: np.ndarray          # (n, 3)
    ang: np.ndarray          # (n, 3)
    mass: np.ndarray         # (n,)
    inertia: np.ndarray      # (n, 9) row-major body-frame inertia
    shape: np.ndarray        # (n,) uint32 global shape index
    flags: np.ndarray        # (n,) uint32
    shape_type: np.ndarray   # (n_shapes,) uint32 (0 box, 1 sphere)
    shape_half: np.ndarray   # (n_shapes, 3) float32
    body_offset: np.ndarray  # (n_scenes + 1,) uint32
    shape_offset: np.ndarray  # (n_scenes + 1,) uint32
    bounds: np.ndarray       # (n_scenes, 6) float32
    targets: np.ndarray      # (n, 3) float32
    max_pairs: int
    max_contacts: int
    dt: float
    n_iters: int
    friction: float
    gravity: tuple = (0.0, -9.81, 0.0)
    n_substeps: int = 1
    meta: dict = field(default_factory=dict)

    @property
    def n_bodies(self) -> int:
        return int(self.mass.shape[0])

    @property
    def n_scenes(self) -> int:
        return int(self.body_offset.shape[0] - 1)

    def scene(self, s: int) -> "SceneSet":
        """Scene s as a stand-alone set with local body and shape indices."""
        b0, b1 = int(self.body_offset[s]), int(self.body_offset[s + 1])
        s0, s1 = int(self.shape_offset[s]), int(self.shape_offset[s + 1])
        n = b1 - b0
        return SceneSet(
            pos=self.pos[b0:b1].copy(), rot=self.rot[b0:b1].copy(), vel=self.vel[b0:b1].copy(),
            ang=self.ang[b0:b1].copy(), mass=self.mass[b0:b1].copy(), inertia=self.inertia[b0:b1].copy(),
            shape=(self.shape[b0:b1] - s0).astype(np.uint32), flags=self.flags[b0:b1].copy(),
            shape_type=self.shape_type[s0:s1].copy(), shape_half=self.shape_half[s0:s1].copy(),
            body_offset=np.array([0, n], np.uint32), shape_offset=np.array([0, s1 - s0], np.uint32),
            bounds=self.bounds[s:s + 1].copy(), targets=self.targets[b0:b1].copy(),
            max_pairs=max(64, 48 * n + 64), max_contacts=max(64, 16 * n + 64), dt=self.dt,
            n_iters=self.n_iters, friction=self.friction, gravity=self.gravity, n_substeps=self.n_substeps,
        )


def make(kind: int, seed: int = 1, a0: int = 0, a1: int = 0, a2: int = 0, spacing: float = 1.0,
         jitter: float = 0.0, builder=None) -> SceneSet:
    lib, prefix = builder if builder is not None else (load_library(), "dyph")
    fn = getattr(lib, prefix + "_scene_make")
    fn.restype = ctypes.POINTER(_SceneSetC)
    fn.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                   ctypes.c_float, ctypes.c_float]
    p = fn(kind, seed, a0, a1, a2, spacing, jitter)
    if not p:
        raise ValueError(f"dyph_scene_make rejected kind={kind} a=({a0},{a1},{a2})")
    c = p.contents
    n, ns, nsc = c.n_bodies, c.n_shapes, c.n_scenes

    def arr(ptr, count, dt, shape=None):
        a = np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)
        return a.reshape(shape) if shape else a

    out = SceneSet(
        pos=arr(c.pos, 3 * n, np.float32, (n, 3)), rot=arr(c.rot, 4 * n, np.float32, (n, 4)),
        vel=arr(c.vel, 3 * n, np.float32, (n, 3)), ang=arr(c.ang, 3 * n, np.float32, (n, 3)),
        mass=arr(c.mass, n, np.float32), inertia=arr(c.inertia, 9 * n, np.float32, (n, 9)),
        shape=arr(c.shape, n, np.uint32), flags=arr(c.flags, n, np.uint32),
        shape_type=arr(c.shape_type, ns, np.uint32), shape_half=arr(c.shape_half, 3 * ns, np.float32, (ns, 3)),
        body_offset=arr(c.body_offset, nsc + 1, np.uint32), shape_offset=arr(c.shape_offset, nsc + 1, np.uint32),
        bounds=arr(c.bounds, 6 * nsc, np.float32, (nsc, 6)), targets=arr(c.targets, 3 * n, np.float32, (n, 3)),
        max_pairs=int(c.max_pairs), max_contacts=int(c.max_contacts), dt=float(c.dt), n_iters=int(c.n_iters),
        friction=float(c.friction), meta={"kind": kind, "seed": seed, "a": (a0, a1, a2),
                                          "spacing": spacing, "jitter": jitter},
    )
    free = getattr(lib, prefix + "_scene_free")
    free.argtypes = [ctypes.POINTER(_SceneSetC)]
    free(p)
    return out


def stress_blocks(spacing: float = 0.85, jitter: float = 0.01, seed: int = 1, grid=(8, 16, 8),
                  builder=None) -> SceneSet:
    """1024 boxes on an 8 x 8 footprint, 16 high, over the 20 x 0.5 x 20 ground."""
    return make(BOX_GRID, seed, grid[0], grid[1], grid[2], spacing, jitter, builder=builder)


def determinism(grid=(2, 2, 2), builder=None) -> SceneSet:
    """The reference's sim-determinism scene (8 boxes + ground by default)."""
    return make(DETERMINISM, 0, grid[0], grid[1], grid[2], 1.0, 0.0, builder=builder)


def random_pile(n: int = 65536, seed: int = 2, builder=None) -> SceneSet:
    return make(RANDOM_PILE, seed, n, builder=builder)


def batch(n_scenes: int = 4096, lo: int = 8, hi: int = 256, seed: int = 3, builder=None) -> SceneSet:
    return make(BATCH, seed, n_scenes, lo, hi, builder=builder)


def push(n_scenes: int = 256, seed: int = 4, builder=None) -> SceneSet:
    return make(PUSH, seed, n_scenes, builder=builder)


def batch_mixed(n_scenes: int = 1024, lo: int = 16, hi: int = 512, seed: int = 5, builder=None) -> SceneSet:
    return make(BATCH_MIXED, seed, n_scenes, lo, hi, builder=builder)
