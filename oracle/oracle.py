"""ctypes access to the two CPU checkers (test infrastructure only).

``Checker("oracle")`` loads the plain-C restatement (oracle/_build), and
``Checker("ref")`` loads the reference's own sources built on the host SYCL
shim (oracle/_ref). Both expose the interface of oracle/oracle_api.h.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libdyphur_oracle.so")
FP64_SO = os.path.join(HERE, "_build", "libdyphur_fp64.so")
DUAL_SO = os.path.join(HERE, "_build", "libdyphur_dual.so")
REF_SO = os.path.join(HERE, "_ref", "libdyphur_ref.so")

STAGE_INTEGRATE, STAGE_BROADPHASE, STAGE_NARROWPHASE, STAGE_SOLVE = 1, 2, 3, 4
SOLVER_REFERENCE, SOLVER_SERIAL, SOLVER_COLORED = 0, 1, 2


class _Scene(ctypes.Structure):
    _fields_ = [
        ("n_bodies", ctypes.c_uint32), ("pos", ctypes.c_void_p), ("rot", ctypes.c_void_p),
        ("vel", ctypes.c_void_p), ("ang", ctypes.c_void_p), ("mass", ctypes.c_void_p),
        ("inertia", ctypes.c_void_p), ("shape", ctypes.c_void_p), ("flags", ctypes.c_void_p),
        ("n_shapes", ctypes.c_uint32), ("shape_type", ctypes.c_void_p), ("shape_half", ctypes.c_void_p),
        ("max_pairs", ctypes.c_uint32), ("max_contacts", ctypes.c_uint32), ("n_iters", ctypes.c_int32),
        ("friction", ctypes.c_float), ("bounds", ctypes.c_float * 6), ("gravity", ctypes.c_float * 3),
        ("dt", ctypes.c_float), ("n_substeps", ctypes.c_int32),
    ]


def build_oracle() -> str:
    """Compile the C restatement if needed (gcc only; works on any host)."""
    srcs = [os.path.join(HERE, f) for f in ("dyphur_oracle.c", "dual_oracle.cpp")]
    stale = any(not os.path.exists(so) for so in (ORACLE_SO, DUAL_SO, FP64_SO)) or \
        os.path.getmtime(ORACLE_SO) < os.path.getmtime(srcs[0]) or \
        min(os.path.getmtime(DUAL_SO), os.path.getmtime(FP64_SO)) < os.path.getmtime(srcs[1])
    if stale:
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


PARAM_VEL, PARAM_ANG, PARAM_INV_MASS = 0, 3, 6


def dual_rollout(state13, inv_mass, iI6, shape_type, half3, flags, n_frames, dt, gravity, n_substeps, n_iters, mu,
                 params, targets, mask, at_float=False, shift_param=-1, shift=0.0):
    """FP64 forward-mode gradient of L = Σ_{mask} |x_final - target|^2 over one
    scene stepped n_frames frames in the sequential order (oracle/dual_oracle.cpp),
    along the float run's contact set and branches; at_float takes the chain
    rule's coefficients at the float values (the FP64 derivative of the float map);
    shift_param / shift move one parameter's FP64 value only (for central differences
    of the FP64 re-run along the same branches).
    params: list of (kind, body), kind 0-2 velocity x/y/z, 3-5 spin x/y/z, 6 inverse mass.
    Returns (loss, grad [len(params)], final float state [13, n], final FP64 state [13, n])."""
    build_oracle()
    L = ctypes.CDLL(DUAL_SO)
    f = L.dyd_rollout
    f.restype = ctypes.c_int
    n = int(np.asarray(inv_mass).shape[0])
    arrs = [np.ascontiguousarray(state13, np.float32), np.ascontiguousarray(inv_mass, np.float32),
            np.ascontiguousarray(iI6, np.float32), np.ascontiguousarray(shape_type, np.uint32),
            np.ascontiguousarray(half3, np.float32), np.ascontiguousarray(flags, np.uint32),
            np.ascontiguousarray(gravity, np.float32)]
    kind = np.ascontiguousarray([k for k, _ in params], np.int32)
    body = np.ascontiguousarray([b for _, b in params], np.uint32)
    tgt = np.ascontiguousarray(targets, np.float32).reshape(-1)
    msk = np.ascontiguousarray(mask, np.uint8)
    loss = ctypes.c_double()
    grad = np.zeros(len(params), np.float64)
    fin_f = np.zeros((13, n), np.float32)
    fin_v = np.zeros((13, n), np.float64)
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_uint32] + [vp] * 6 + [ctypes.c_int, ctypes.c_float, vp, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_float, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_double, vp, vp, vp, vp]
    rc = f(n, *[a.ctypes.data for a in arrs[:6]], int(n_frames), float(dt), arrs[6].ctypes.data, int(n_substeps),
           int(n_iters), float(mu), len(params), kind.ctypes.data, body.ctypes.data, tgt.ctypes.data,
           msk.ctypes.data, int(bool(at_float)), int(shift_param), float(shift), ctypes.byref(loss),
           grad.ctypes.data, fin_f.ctypes.data, fin_v.ctypes.data)
    if rc != 0:
        raise ValueError("too many gradient parameters for the dual-number oracle")
    return loss.value, grad, fin_f, fin_v


def fp64_run(state13, inv_mass, iI6, shape_type, half3, flags, n_frames, dt, gravity, n_substeps, n_iters, mu,
             mode=SOLVER_SERIAL, local=True):
    """FP64 re-run of one scene's frame step along the float run's decisions
    (oracle/dual_oracle.cpp, dyd_fp64_run) in solver order `mode` (0 the
    reference's, 1 serial, 2 coloured). local: each frame's FP64 run starts
    from the float state (the frame's own rounding error); otherwise the FP64
    state is carried (the accumulated error, which contact-rich scenes amplify
    without bound). Returns (err_pos [n_frames] = max |x_float - x_fp64| per
    frame in m, err_rot [n_frames] = max quaternion component error, final
    float state [13, n], final FP64 state [13, n])."""
    build_oracle()
    L = ctypes.CDLL(FP64_SO)
    f = L.dyd_fp64_run
    f.restype = ctypes.c_int
    n = int(np.asarray(inv_mass).shape[0])
    arrs = [np.ascontiguousarray(state13, np.float32), np.ascontiguousarray(inv_mass, np.float32),
            np.ascontiguousarray(iI6, np.float32), np.ascontiguousarray(shape_type, np.uint32),
            np.ascontiguousarray(half3, np.float32), np.ascontiguousarray(flags, np.uint32),
            np.ascontiguousarray(gravity, np.float32)]
    ep = np.zeros(n_frames, np.float64)
    er = np.zeros(n_frames, np.float64)
    fin_f = np.zeros((13, n), np.float32)
    fin_v = np.zeros((13, n), np.float64)
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_uint32] + [vp] * 6 + [ctypes.c_int, ctypes.c_float, vp, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_float, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]
    f(n, *[a.ctypes.data for a in arrs[:6]], int(n_frames), float(dt), arrs[6].ctypes.data, int(n_substeps),
      int(n_iters), float(mu), int(mode), int(bool(local)), ep.ctypes.data, er.ctypes.data, fin_f.ctypes.data,
      fin_v.ctypes.data)
    return ep, er, fin_f, fin_v


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def scene_builder(which: str | None = None):
    """(cdll, prefix) of the scene builders inside a checker library, for
    dyphur_b200.scenes(..., builder=...): the reference build's copy when it
    exists, else the C restatement's."""
    which = which or ("ref" if ref_available() else "oracle")
    if which == "ref":
        return ctypes.CDLL(REF_SO), "dyr"
    return ctypes.CDLL(build_oracle()), "dyo"


class Checker:
    def __init__(self, which: str = "oracle"):
        if which == "oracle":
            self.lib = ctypes.CDLL(build_oracle())
            p = "dyo_"
        elif which == "ref":
            if not ref_available():
                raise FileNotFoundError(REF_SO)
            self.lib = ctypes.CDLL(REF_SO)
            p = "dyr_"
        else:
            raise ValueError(which)
        self.which = which
        L = self.lib
        vp, u32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
        self.f_create = getattr(L, p + "create"); self.f_create.restype = vp
        self.f_create.argtypes = [ctypes.POINTER(_Scene)]
        self.f_destroy = getattr(L, p + "destroy"); self.f_destroy.argtypes = [vp]
        self.f_stage = getattr(L, p + "run_stage"); self.f_stage.argtypes = [vp, i32, i32]
        self.f_step = getattr(L, p + "step"); self.f_step.argtypes = [vp, i32, i32]
        self.f_get_state = getattr(L, p + "get_state"); self.f_get_state.argtypes = [vp, vp]
        self.f_set_state = getattr(L, p + "set_state"); self.f_set_state.argtypes = [vp, vp]
        self.f_get_inv = getattr(L, p + "get_inv"); self.f_get_inv.argtypes = [vp, vp, vp]
        self.f_hash = getattr(L, p + "hash"); self.f_hash.restype = ctypes.c_uint64
        self.f_hash.argtypes = [vp]
        self.f_pairs = getattr(L, p + "get_pairs"); self.f_pairs.restype = u32
        self.f_pairs.argtypes = [vp, vp, u32]
        self.f_contacts = getattr(L, p + "get_contacts"); self.f_contacts.restype = u32
        self.f_contacts.argtypes = [vp, vp, vp, u32]
        self.f_bvh = getattr(L, p + "get_bvh"); self.f_bvh.argtypes = [vp] * 7
        self.f_colors = getattr(L, p + "get_colors"); self.f_colors.restype = u32
        self.f_colors.argtypes = [vp, vp, u32]
        self.f_rays = getattr(L, p + "ray_query"); self.f_rays.restype = None
        self.f_rays.argtypes = [vp, vp, u32, vp, vp]
        self.f_sensor = getattr(L, p + "contact_sensor"); self.f_sensor.restype = u32
        self.f_sensor.argtypes = [vp, u32, vp, vp, u32]


class World:
    """One scene stepped by a CPU checker."""

    def __init__(self, scene, which: str = "oracle", max_pairs: int | None = None,
                 max_contacts: int | None = None):
        self.ck = Checker(which)
        s = scene
        self.n = s.n_bodies
        self._keep = [np.ascontiguousarray(a) for a in (
            s.pos.astype(np.float32), s.rot.astype(np.float32), s.vel.astype(np.float32),
            s.ang.astype(np.float32), s.mass.astype(np.float32), s.inertia.astype(np.float32),
            s.shape.astype(np.uint32), s.flags.astype(np.uint32), s.shape_type.astype(np.uint32),
            s.shape_half.astype(np.float32))]
        d = _Scene()
        d.n_bodies = self.n
        for name, a in zip(("pos", "rot", "vel", "ang", "mass", "inertia", "shape", "flags"), self._keep[:8]):
            setattr(d, name, a.ctypes.data)
        d.n_shapes = int(s.shape_type.shape[0])
        d.shape_type = self._keep[8].ctypes.data
        d.shape_half = self._keep[9].ctypes.data
        self.max_pairs = int(max_pairs or s.max_pairs)
        self.max_contacts = int(max_contacts or s.max_contacts)
        d.max_pairs, d.max_contacts = self.max_pairs, self.max_contacts
        d.n_iters, d.friction = int(s.n_iters), float(s.friction)
        d.bounds[:] = [float(x) for x in np.asarray(s.bounds).reshape(-1)[:6]]
        d.gravity[:] = [float(x) for x in s.gravity]
        d.dt, d.n_substeps = float(s.dt), int(s.n_substeps)
        self._desc = d
        self.h = self.ck.f_create(ctypes.byref(d))
        if not self.h:
            raise RuntimeError(f"{which}: create failed")

    def close(self):
        if self.h:
            self.ck.f_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stage(self, st: int, mode: int = SOLVER_REFERENCE) -> int:
        return int(self.ck.f_stage(self.h, st, mode))

    def step(self, frames: int, mode: int = SOLVER_REFERENCE) -> int:
        return int(self.ck.f_step(self.h, frames, mode))

    def state(self) -> np.ndarray:
        out = np.empty((13, self.n), np.float32)
        self.ck.f_get_state(self.h, out.ctypes.data)
        return out

    def set_state(self, st: np.ndarray) -> None:
        st = np.ascontiguousarray(st, dtype=np.float32).reshape(13, self.n)
        self.ck.f_set_state(self.h, st.ctypes.data)

    def inv(self):
        im = np.empty(self.n, np.float32)
        ii = np.empty((6, self.n), np.float32)
        self.ck.f_get_inv(self.h, im.ctypes.data, ii.ctypes.data)
        return im, ii

    def hash(self) -> int:
        return int(self.ck.f_hash(self.h))

    def pairs(self):
        cap = self.max_pairs
        buf = np.empty((cap, 2), np.uint32)
        n = int(self.ck.f_pairs(self.h, buf.ctypes.data, cap))
        return buf[:min(n, cap)].copy(), n

    def contacts(self):
        cap = self.max_contacts
        ab = np.empty((cap, 2), np.uint32)
        p7 = np.empty((cap, 7), np.float32)
        n = int(self.ck.f_contacts(self.h, ab.ctypes.data, p7.ctypes.data, cap))
        m = min(n, cap)
        return ab[:m].copy(), p7[:m].copy()

    def bvh(self):
        n = self.n
        keys = np.zeros(n, np.uint64)
        si = np.zeros(n, np.uint32)
        left = np.zeros(max(n - 1, 1), np.int32)
        right = np.zeros(max(n - 1, 1), np.int32)
        parent = np.zeros(max(2 * n - 1, 1), np.int32)
        aabb = np.zeros((max(2 * n - 1, 1), 8), np.uint16)
        self.ck.f_bvh(self.h, keys.ctypes.data, si.ctypes.data, left.ctypes.data, right.ctypes.data,
                      parent.ctypes.data, aabb.ctypes.data)
        return dict(keys=keys, sorted_idx=si, left=left[:n - 1], right=right[:n - 1],
                    parent=parent[:2 * n - 1], aabb=aabb[:2 * n - 1])

    def ray_query(self, rays: np.ndarray):
        """Closest hits of rays (n, 7) = origin xyz, direction xyz, t_max over
        the tree of the last broadphase stage: (t float32 (n,), body uint32 (n,))."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 7)
        t = np.empty(rays.shape[0], np.float32)
        body = np.empty(rays.shape[0], np.uint32)
        self.ck.f_rays(self.h, rays.ctypes.data, rays.shape[0], t.ctypes.data, body.ctypes.data)
        return t, body

    def contact_sensor(self, shape_idx: int):
        """Contacts of the last narrowphase stage that involve shape_idx:
        (ab (m, 2) uint32, p7 (m, 7) float32) in store order."""
        cap = self.max_contacts
        ab = np.empty((cap, 2), np.uint32)
        p7 = np.empty((cap, 7), np.float32)
        m = int(self.ck.f_sensor(self.h, int(shape_idx), ab.ctypes.data, p7.ctypes.data, cap))
        m = min(m, cap)
        return ab[:m].copy(), p7[:m].copy()

    def colors(self):
        cap = self.max_contacts
        buf = np.empty(cap, np.uint32)
        n = int(self.ck.f_colors(self.h, buf.ctypes.data, cap))
        return buf[:min(n, cap)].copy()


def fnv1a64_state(state13: np.ndarray) -> int:
    """FNV-1a-64 of pos_x..rot_z (examples/stress_test_blocks/main.cpp:34-41, 301-311)."""
    data = np.ascontiguousarray(state13[:7], dtype=np.float32).tobytes()
    h = 0xcbf29ce484222325
    for b in data:
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h
