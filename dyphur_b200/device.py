"""Device-resident scenes and the frame-step handles, over the C ABI.

PyTorch provides the device memory (CUDA tensors) and streams; every kernel
that runs is the library's own (``libdyphur_b200.so``). There is no CPU path:
constructing any of these objects without a B200 raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .capi import check

STATE_FIELDS = ("pos_x", "pos_y", "pos_z", "rot_w", "rot_x", "rot_y", "rot_z",
                "vel_x", "vel_y", "vel_z", "ang_x", "ang_y", "ang_z")
INV_FIELDS = ("iI_xx", "iI_yy", "iI_zz", "iI_xy", "iI_xz", "iI_yz")


def require_device() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("dyphur_b200 needs a CUDA device (sm_100); none is visible")
    check(capi.lib().dyph_device_check(), "dyph_device_check")


def _ptr(t: torch.Tensor) -> int:
    return int(t.data_ptr())


def pack_bodies(scene):
    """Host BodyStore::add over a SceneSet -> (state13, inv_mass, iI6, flags)."""
    n = scene.n_bodies
    st = np.empty((13, n), np.float32)
    im = np.empty(n, np.float32)
    ii = np.empty((6, n), np.float32)
    fl = np.empty(n, np.uint32)
    args = [np.ascontiguousarray(a) for a in (scene.pos.astype(np.float32), scene.rot.astype(np.float32),
                                              scene.vel.astype(np.float32), scene.ang.astype(np.float32),
                                              scene.mass.astype(np.float32), scene.inertia.astype(np.float32),
                                              scene.flags.astype(np.uint32))]
    capi.lib().dyph_pack_bodies(n, *[a.ctypes.data for a in args], st.ctypes.data, im.ctypes.data,
                                ii.ctypes.data, fl.ctypes.data)
    return st, im, ii, fl


class DeviceBodies:
    """BodyView SoA in CUDA memory (one tensor per field)."""

    def __init__(self, scene, device="cuda"):
        require_device()
        st, im, ii, fl = pack_bodies(scene)
        self.n = scene.n_bodies
        # one allocation for the float fields keeps them 256-byte aligned and contiguous
        pad = (self.n + 63) // 64 * 64
        self.fbuf = torch.zeros((20, pad), dtype=torch.float32, device=device)
        self.fbuf[:13, :self.n] = torch.from_numpy(st).to(device)
        self.fbuf[13, :self.n] = torch.from_numpy(im).to(device)
        self.fbuf[14:20, :self.n] = torch.from_numpy(ii).to(device)
        self.shape = torch.from_numpy(scene.shape.astype(np.int32)).to(device)
        self.flags = torch.from_numpy(fl.astype(np.int32)).to(device)
        self.view = capi.Bodies()
        for k, f in enumerate(STATE_FIELDS):
            setattr(self.view, f, _ptr(self.fbuf[k]))
        self.view.inv_mass = _ptr(self.fbuf[13])
        for k, f in enumerate(INV_FIELDS):
            setattr(self.view, f, _ptr(self.fbuf[14 + k]))
        self.view.shape = _ptr(self.shape)
        self.view.flags = _ptr(self.flags)
        self.view.n = self.n

    def state(self) -> np.ndarray:
        return self.fbuf[:13, :self.n].cpu().numpy().copy()

    def set_state(self, st: np.ndarray) -> None:
        self.fbuf[:13, :self.n] = torch.from_numpy(np.ascontiguousarray(st, np.float32)).to(self.fbuf.device)

    def inv(self):
        return self.fbuf[13, :self.n].cpu().numpy(), self.fbuf[14:20, :self.n].cpu().numpy()


class DeviceShapes:
    def __init__(self, scene, device="cuda"):
        self.n = int(scene.shape_type.shape[0])
        self.type = torch.from_numpy(scene.shape_type.astype(np.int32)).to(device)
        self.half = torch.from_numpy(np.ascontiguousarray(scene.shape_half.T, np.float32)).to(device)
        self.ext = torch.zeros(max(self.n, 1), dtype=torch.int32, device=device)
        self.view = capi.Shapes(_ptr(self.type), _ptr(self.half[0]), _ptr(self.half[1]), _ptr(self.half[2]),
                                _ptr(self.ext), self.n)


def _stream_ptr(stream) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def aabb(bounds) -> capi.AABB:
    b = [float(x) for x in np.asarray(bounds).reshape(-1)[:6]]
    return capi.AABB(*b)


class Broadphase:
    """Mirror of class Broadphase (core/include/core/broadphase.hpp:50-111)."""

    def __init__(self, max_bodies: int, max_pairs: int):
        require_device()
        h = C.c_void_p()
        check(capi.lib().dyph_broadphase_create(max_bodies, max_pairs, C.byref(h)), "dyph_broadphase_create")
        self.h = h
        self.max_pairs = max_pairs

    def __del__(self):
        if getattr(self, "h", None):
            capi.lib().dyph_broadphase_destroy(self.h)
            self.h = None

    def build_and_query(self, bodies: DeviceBodies, shapes: DeviceShapes, bounds, stream=None) -> None:
        b = aabb(bounds)
        check(capi.lib().dyph_broadphase_build_and_query(self.h, C.byref(bodies.view), C.byref(shapes.view),
                                                         C.byref(b), _stream_ptr(stream)), "build_and_query")

    def download_count(self, stream=None) -> int:
        out = C.c_uint32()
        check(capi.lib().dyph_broadphase_download_count(self.h, _stream_ptr(stream), C.byref(out)))
        return int(out.value)

    def pairs(self, stream=None) -> np.ndarray:
        n = min(self.download_count(stream), self.max_pairs)
        out = np.empty((n, 2), np.uint32)
        if n:
            torch.cuda.synchronize()
            host = torch.empty((n, 2), dtype=torch.int32)
            src = capi.lib().dyph_broadphase_pairs(self.h)
            _d2h(host, src, n * 8)
            out = host.numpy().view(np.uint32).copy()
        return out

    def bvh_view(self, n: int) -> capi.BvhView:
        v = capi.BvhView()
        check(capi.lib().dyph_broadphase_bvh_view(self.h, n, C.byref(v)))
        return v

    def bvh(self, n: int) -> dict:
        v = capi.BvhView()
        check(capi.lib().dyph_broadphase_bvh_view(self.h, n, C.byref(v)))
        out = {}
        specs = [("keys", v.sorted_keys, n, np.uint64, torch.int64), ("sorted_idx", v.sorted_idx, n, np.uint32, torch.int32),
                 ("left", v.left, n - 1, np.int32, torch.int32), ("right", v.right, n - 1, np.int32, torch.int32),
                 ("parent", v.parent, 2 * n - 1, np.int32, torch.int32)]
        torch.cuda.synchronize()
        for name, ptr, cnt, npdt, tdt in specs:
            host = torch.empty(max(cnt, 0), dtype=tdt)
            if cnt > 0:
                _d2h(host, ptr, cnt * host.element_size())
            out[name] = host.numpy().view(npdt).copy()
        box = torch.empty((2 * n - 1, 8), dtype=torch.int16)
        _d2h(box, v.aabb, (2 * n - 1) * 16)
        out["aabb"] = box.numpy().view(np.uint16).copy()
        return out


def _d2h(host: torch.Tensor, dev_ptr, nbytes: int) -> None:
    """Blocking device -> host copy of raw bytes (dyph_copy_to_host)."""
    if nbytes <= 0:
        return
    check(capi.lib().dyph_copy_to_host(host.data_ptr(), int(dev_ptr), nbytes, None), "dyph_copy_to_host")


def _h2d(dev_ptr, host: torch.Tensor, nbytes: int) -> None:
    if nbytes <= 0:
        return
    check(capi.lib().dyph_copy_to_device(int(dev_ptr), host.data_ptr(), nbytes, None), "dyph_copy_to_device")


def read_contacts(view: capi.Contacts, n: int):
    """Download the first n rows of a ContactView: (ab [n,2] u32, p7 [n,7] f32)."""
    torch.cuda.synchronize()
    ab = np.empty((n, 2), np.uint32)
    p7 = np.empty((n, 7), np.float32)
    if n == 0:
        return ab, p7
    cols = [view.body_a, view.body_b, view.pos_x, view.pos_y, view.pos_z, view.norm_x, view.norm_y, view.norm_z,
            view.depth]
    for k, ptr in enumerate(cols):
        host = torch.empty(n, dtype=torch.int32 if k < 2 else torch.float32)
        _d2h(host, ptr, n * 4)
        if k < 2:
            ab[:, k] = host.numpy().view(np.uint32)
        else:
            p7[:, k - 2] = host.numpy()
    return ab, p7


class Narrowphase:
    """Mirror of class Narrowphase (core/include/core/narrowphase.hpp:26-73)."""

    def __init__(self, max_contacts: int):
        require_device()
        h = C.c_void_p()
        check(capi.lib().dyph_narrowphase_create(max_contacts, C.byref(h)), "dyph_narrowphase_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            capi.lib().dyph_narrowphase_destroy(self.h)
            self.h = None

    def run(self, bp: Broadphase, bodies: DeviceBodies, shapes: DeviceShapes, stream=None) -> None:
        L = capi.lib()
        check(L.dyph_narrowphase_run(self.h, L.dyph_broadphase_pairs(bp.h), L.dyph_broadphase_count_ptr(bp.h),
                                     C.byref(bodies.view), C.byref(shapes.view), _stream_ptr(stream)), "run")

    def run_pairs(self, pairs_dev: torch.Tensor, n_pairs: int, bodies, shapes, stream=None) -> None:
        check(capi.lib().dyph_narrowphase_run_host_count(self.h, _ptr(pairs_dev), n_pairs, C.byref(bodies.view),
                                                        C.byref(shapes.view), _stream_ptr(stream)), "run")

    def contacts_view(self) -> capi.Contacts:
        v = capi.Contacts()
        check(capi.lib().dyph_narrowphase_contacts(self.h, C.byref(v)))
        return v

    def download_count(self, stream=None):
        a, b = C.c_uint32(), C.c_uint32()
        check(capi.lib().dyph_narrowphase_download_count(self.h, _stream_ptr(stream), C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def contacts(self, stream=None):
        n, _ = self.download_count(stream)
        return read_contacts(self.contacts_view(), n)


def ray_query(bvh: capi.BvhView, bodies: DeviceBodies, shapes: DeviceShapes, rays, stream=None):
    """ray_query (core/include/core/ray_query.hpp:34-40) over a built tree.

    rays: (n, 7) origin xyz, direction xyz, t_max (numpy or a CUDA float32
    tensor). Returns (t, body) as CUDA tensors (float32, int32 holding the
    uint32 body index; -1 = UINT32_MAX = miss)."""
    r = torch.as_tensor(rays, dtype=torch.float32)
    r = r.reshape(-1, 7).to("cuda").contiguous()
    n = r.shape[0]
    hits = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    check(capi.lib().dyph_ray_query(C.byref(bvh), C.byref(bodies.view), C.byref(shapes.view), _ptr(r),
                                    _ptr(hits), n, _stream_ptr(stream)), "dyph_ray_query")
    return hits[:, 0].view(torch.float32), hits[:, 1]


class ContactSensor:
    """Mirror of class ContactSensor (core/include/core/contact_sensor.hpp:20-58):
    contacts involving one shape, filtered on the device."""

    def __init__(self, shape_idx: int):
        require_device()
        h = C.c_void_p()
        check(capi.lib().dyph_contact_sensor_create(int(shape_idx), C.byref(h)), "dyph_contact_sensor_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            capi.lib().dyph_contact_sensor_destroy(self.h)
            self.h = None

    def query(self, contacts: capi.Contacts, bodies: DeviceBodies, stream=None) -> int:
        out = C.c_uint32()
        check(capi.lib().dyph_contact_sensor_query(self.h, C.byref(contacts), bodies.view.shape, bodies.n,
                                                   _stream_ptr(stream), C.byref(out)), "dyph_contact_sensor_query")
        return int(out.value)

    def count(self) -> int:
        return int(capi.lib().dyph_contact_sensor_count(self.h))

    def shape_idx(self) -> int:
        return int(capi.lib().dyph_contact_sensor_shape_idx(self.h))

    def rows(self):
        """(ab (m, 2) uint32, p7 (m, 7) float32) of the last query, copied from
        the sensor's pinned host arrays."""
        v = capi.Contacts()
        check(capi.lib().dyph_contact_sensor_host_view(self.h, C.byref(v)))
        m = self.count()
        ab = np.empty((m, 2), np.uint32)
        p7 = np.empty((m, 7), np.float32)
        if m:
            cols = [v.body_a, v.body_b, v.pos_x, v.pos_y, v.pos_z, v.norm_x, v.norm_y, v.norm_z, v.depth]
            for k, ptr in enumerate(cols):
                a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint32)), shape=(m,))
                if k < 2:
                    ab[:, k] = a
                else:
                    p7[:, k - 2] = a.view(np.float32)
        return ab, p7


class XpbdSolver:
    """Mirror of class XpbdSolver (core/include/core/xpbd_solver.hpp:29-70)."""

    def __init__(self, n_iters: int = 10, max_contacts: int = 16384, max_bodies: int = 1 << 16,
                 friction: float = 0.5):
        require_device()
        h = C.c_void_p()
        check(capi.lib().dyph_xpbd_create(n_iters, max_contacts, max_bodies, friction, C.byref(h)),
              "dyph_xpbd_create")
        self.h = h
        self.max_contacts = max_contacts

    def __del__(self):
        if getattr(self, "h", None):
            capi.lib().dyph_xpbd_destroy(self.h)
            self.h = None

    def set_mode(self, mode: int) -> None:
        check(capi.lib().dyph_xpbd_set_mode(self.h, mode))

    def set_force_serial(self, v: bool) -> None:
        self.set_mode(capi.SOLVER_SEQUENTIAL if v else capi.SOLVER_REFERENCE)

    def solve(self, contacts: capi.Contacts, bodies: DeviceBodies, dt: float, stream=None) -> None:
        check(capi.lib().dyph_xpbd_solve(self.h, C.byref(contacts), C.byref(bodies.view), float(dt),
                                         _stream_ptr(stream)), "solve")

    def colors(self, n: int, stream=None):
        out = np.empty(max(n, 1), np.uint32)
        nc = C.c_uint32()
        check(capi.lib().dyph_xpbd_download_colors(self.h, _stream_ptr(stream), out.ctypes.data_as(capi._up), n,
                                                   C.byref(nc)))
        return out[:n], int(nc.value)


def integrate(bodies: DeviceBodies, gravity=(0.0, -9.81, 0.0), dt=1.0 / 60.0, n_substeps=1, stream=None) -> None:
    p = capi.IntegratorParams((C.c_float * 3)(*gravity), dt, n_substeps)
    check(capi.lib().dyph_integrate(C.byref(bodies.view), C.byref(p), _stream_ptr(stream)), "integrate")


def device_error(stream=None) -> int:
    code = C.c_uint32()
    check(capi.lib().dyph_download_device_error(_stream_ptr(stream), C.byref(code)))
    return int(code.value)


def device_error_site(stream=None) -> tuple:
    """(code, site) of the first device-side error since the last read; both cleared."""
    code, site = C.c_uint32(), C.c_uint32()
    check(capi.lib().dyph_download_device_error_site(_stream_ptr(stream), C.byref(code), C.byref(site)))
    return int(code.value), int(site.value)


def set_spin_limit(limit: int) -> None:
    """Iteration limit of every bounded device wait (0 = the default)."""
    check(capi.lib().dyph_set_spin_limit(int(limit)), "dyph_set_spin_limit")


def wait_selftest(which: int, stream=None) -> None:
    """A bounded wait that nothing ends (1 look-back, 3 grid barrier)."""
    check(capi.lib().dyph_wait_selftest(int(which), _stream_ptr(stream)), "dyph_wait_selftest")


def check_finite(bodies: DeviceBodies, stream=None) -> tuple:
    """(status, first bad body index) of dyph_bodies_check_finite."""
    first = C.c_uint32()
    st = capi.lib().dyph_bodies_check_finite(C.byref(bodies.view), _stream_ptr(stream), C.byref(first))
    if st not in (capi.OK, capi.ERR_NOT_FINITE):
        check(st, "dyph_bodies_check_finite")
    return int(st), int(first.value)


def state_hash(bodies: DeviceBodies, stream=None) -> int:
    out = torch.zeros(1, dtype=torch.int64, device=bodies.fbuf.device)
    check(capi.lib().dyph_fnv1a64_state(C.byref(bodies.view), _ptr(out), _stream_ptr(stream)))
    return int(out.cpu().numpy().view(np.uint64)[0])


class World:
    """The whole frame step on one scene (dyph_world_*), graph-replayed."""

    def __init__(self, scene, mode: int = capi.SOLVER_REFERENCE, max_pairs=None, max_contacts=None):
        require_device()
        self.scene = scene
        self.bodies = DeviceBodies(scene)
        self.shapes = DeviceShapes(scene)
        d = capi.WorldDesc()
        d.bodies = self.bodies.view
        d.shapes = self.shapes.view
        d.scene_bounds = aabb(scene.bounds[0])
        d.integrator = capi.IntegratorParams((C.c_float * 3)(*scene.gravity), scene.dt, scene.n_substeps)
        if scene.n_scenes > 1:  # capacities for all scenes together
            max_pairs = max_pairs or 48 * scene.n_bodies + 64 * scene.n_scenes
            max_contacts = max_contacts or 16 * scene.n_bodies + 64 * scene.n_scenes
        d.max_pairs = int(max_pairs or scene.max_pairs)
        d.max_contacts = int(max_contacts or scene.max_contacts)
        d.n_iters = scene.n_iters
        d.friction = scene.friction
        d.mode = mode
        self.desc = d
        h = C.c_void_p()
        check(capi.lib().dyph_world_create(C.byref(d), None, C.byref(h)), "dyph_world_create")
        self.h = h
        if scene.n_scenes > 1:
            # Batched scenes: one tree over all scenes, pairs kept inside each scene.
            off = np.ascontiguousarray(scene.body_offset, np.uint32)
            bnds = (capi.AABB * scene.n_scenes)(*[aabb(b) for b in scene.bounds])
            self._scene_offset = off
            check(capi.lib().dyph_world_set_scenes(h, scene.n_scenes, off.ctypes.data, bnds),
                  "dyph_world_set_scenes")
        # the state at creation (rows pos, rot, vel, ang), the start of differentiable rollouts
        self.initial = self.bodies.fbuf[:13].clone()
        bp, np_, sv = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(capi.lib().dyph_world_broadphase(h, C.byref(bp)))
        check(capi.lib().dyph_world_narrowphase(h, C.byref(np_)))
        check(capi.lib().dyph_world_solver(h, C.byref(sv)))
        self._bp, self._np, self._sv = bp, np_, sv

    def close(self):
        if getattr(self, "h", None):
            capi.lib().dyph_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, frames: int = 1, stream=None) -> None:
        check(capi.lib().dyph_world_step(self.h, frames, _stream_ptr(stream)), "dyph_world_step")

    def set_trajectory(self, host: torch.Tensor | None, every: int = 2) -> None:
        """Record every `every`-th frame's poses into a pinned host float tensor of shape
        (records, n, 7) (dyph_world_set_trajectory); None stops recording."""
        if host is None:
            check(capi.lib().dyph_world_set_trajectory(self.h, None, 0, 0), "dyph_world_set_trajectory")
            self._traj = None
            return
        if not host.is_pinned() or host.dtype != torch.float32 or host.shape[1:] != (self.bodies.n, 7):
            raise ValueError("trajectory buffer must be a pinned float32 tensor of shape (records, n, 7)")
        check(capi.lib().dyph_world_set_trajectory(self.h, host.data_ptr(), every, host.shape[0]),
              "dyph_world_set_trajectory")
        self._traj = host

    def capture_episode(self, n_frames: int, probe_stage: int = -1) -> None:
        """Record n_frames frames as one graph; probe_stage 0..3 times that stage per frame
        (4: the solver's dataflow kernel alone)."""
        L = capi.lib()
        self._free_probe()
        if probe_stage >= 0:
            evs = []
            for _ in range(2 * n_frames):
                e = C.c_void_p()
                check(L.dyph_event_create(C.byref(e)))
                evs.append(e.value)
            self._probe = ((C.c_void_p * n_frames)(*evs[:n_frames]), (C.c_void_p * n_frames)(*evs[n_frames:]))
            check(L.dyph_world_capture_episode(self.h, n_frames, probe_stage, self._probe[0], self._probe[1]))
        else:
            check(L.dyph_world_capture_episode(self.h, n_frames, -1, None, None))
        self.episode_frames = n_frames

    def history(self, cap: int = 4096):
        """(pairs, contacts) true counts of the most recent frames, oldest first."""
        p = np.zeros(cap, np.uint32)
        c = np.zeros(cap, np.uint32)
        tot = C.c_uint32()
        check(capi.lib().dyph_world_download_history(self.h, None, p.ctypes.data, c.ctypes.data, cap,
                                                     C.byref(tot)))
        m = min(cap, int(tot.value), 4096)
        return p[:m], c[:m]

    def run_episode(self, stream=None) -> None:
        check(capi.lib().dyph_world_run_episode(self.h, _stream_ptr(stream)), "dyph_world_run_episode")

    def probe_ms(self) -> np.ndarray:
        """Per-frame duration (ms) of the probed stage in the last episode run."""
        out = np.zeros(self.episode_frames, np.float64)
        ms = C.c_float()
        for f in range(self.episode_frames):
            check(capi.lib().dyph_event_elapsed_ms(self._probe[0][f], self._probe[1][f], C.byref(ms)))
            out[f] = ms.value
        return out

    def _free_probe(self):
        p = getattr(self, "_probe", None)
        if p:
            for arr in p:
                for e in arr:
                    capi.lib().dyph_event_destroy(e)
        self._probe = None

    def stats(self, stream=None) -> dict:
        v = [C.c_uint32() for _ in range(5)]
        check(capi.lib().dyph_world_download_stats(self.h, _stream_ptr(stream), *[C.byref(x) for x in v]))
        keys = ("last_pairs", "last_contacts", "peak_pairs", "peak_contacts", "status")
        return {k: int(x.value) for k, x in zip(keys, v)}

    def state(self) -> np.ndarray:
        torch.cuda.synchronize()
        return self.bodies.state()

    def hash(self) -> int:
        return state_hash(self.bodies)

    def scene_hashes(self, stream=None) -> np.ndarray:
        """FNV-1a-64 of every scene's poses (uint64 array, one per scene)."""
        n = self.scene.n_scenes
        out = np.zeros(n, np.uint64)
        check(capi.lib().dyph_world_scene_hashes(self.h, _stream_ptr(stream), out.ctypes.data, n))
        return out

    def phase_timing(self, on: bool = True) -> None:
        """Time the phases of fused batched frames (dyph_world_set_phase_timing)."""
        check(capi.lib().dyph_world_set_phase_timing(self.h, int(on)), "dyph_world_set_phase_timing")

    def phase_ns(self) -> np.ndarray:
        """Summed ns of the fused frames' phases since the last read: staging + integrate + boxes,
        pair search, narrowphase, solve set-up (lists, colours or levels, groups), sweep +
        renormalisation, write-back."""
        out = np.zeros(6, np.uint64)
        check(capi.lib().dyph_world_download_phase_ns(self.h, None, out.ctypes.data, 6), "phase_ns")
        return out

    def sync_lists(self) -> None:
        """Compact the last frame's per-scene pair / contact lists (fused batched frames)."""
        check(capi.lib().dyph_world_sync_lists(self.h, None), "dyph_world_sync_lists")

    def pairs(self) -> np.ndarray:
        L = capi.lib()
        self.sync_lists()
        n = C.c_uint32()
        check(L.dyph_broadphase_download_count(self._bp, None, C.byref(n)))
        m = min(int(n.value), int(L.dyph_broadphase_max_pairs(self._bp)))
        host = torch.empty((m, 2), dtype=torch.int32)
        _d2h(host, L.dyph_broadphase_pairs(self._bp), m * 8)
        return host.numpy().view(np.uint32).copy()

    def contacts(self):
        self.sync_lists()
        v = capi.Contacts()
        check(capi.lib().dyph_narrowphase_contacts(self._np, C.byref(v)))
        a, b = C.c_uint32(), C.c_uint32()
        check(capi.lib().dyph_narrowphase_download_count(self._np, None, C.byref(a), C.byref(b)))
        return read_contacts(v, int(a.value))

    def fused_config(self) -> dict:
        """Knobs of the fused batched frame in force (dyph_world_fused_config)."""
        c = capi.FusedConfig()
        check(capi.lib().dyph_world_fused_config(self.h, C.byref(c)), "dyph_world_fused_config")
        return {k: getattr(c, k) for k, _ in capi.FusedConfig._fields_}

    def set_fused_config(self, smem_cap: int, teams: int = 2, register_blocks: int = 0) -> None:
        """teams: 0 every scene a block, 1 small scenes one per warp, 2 also mid-size scenes on two warps."""
        check(capi.lib().dyph_world_set_fused_config(self.h, int(smem_cap), int(teams), int(register_blocks)),
              "dyph_world_set_fused_config")

    def adjoint_config(self) -> dict:
        """Layout of the adjoint's reverse kernel (dyph_world_adjoint_config)."""
        c = capi.FusedConfig()
        check(capi.lib().dyph_world_adjoint_config(self.h, C.byref(c)), "dyph_world_adjoint_config")
        return {k: getattr(c, k) for k, _ in capi.FusedConfig._fields_}

    def set_adjoint_config(self, smem_bytes: int = 0, teams: int = 2) -> None:
        """smem_bytes 0: a third of an SM's shared memory; teams as set_fused_config."""
        check(capi.lib().dyph_world_set_adjoint_config(self.h, int(smem_bytes), int(teams)),
              "dyph_world_set_adjoint_config")

    def autotune(self, frames: int = 16, stream=None) -> dict:
        """Time the fused kernel's configurations from the current state and keep
        the fastest (dyph_world_autotune); returns the chosen configuration."""
        c = capi.FusedConfig()
        check(capi.lib().dyph_world_autotune(self.h, int(frames), _stream_ptr(stream), C.byref(c)),
              "dyph_world_autotune")
        return {k: getattr(c, k) for k, _ in capi.FusedConfig._fields_}

    # The rollout protocol of dyphur_b200.autograd (shared with dyphur_py.World).
    def count(self) -> int:
        return self.bodies.n

    def device_rows(self) -> torch.Tensor:
        return self.bodies.fbuf

    def initial_rows(self) -> torch.Tensor:
        return self.initial

    def rollout_raw(self, frames: int, every: int, d_ckpt: int, stream: int) -> None:
        check(capi.lib().dyph_world_rollout(self.h, frames, every, d_ckpt, stream), "dyph_world_rollout")

    def rollout_backward_raw(self, frames: int, every: int, d_ckpt: int, g_final: int, g_init: int, g_im: int,
                             stream: int) -> None:
        check(capi.lib().dyph_world_rollout_backward(self.h, frames, every, d_ckpt, g_final, g_init, g_im, stream),
              "dyph_world_rollout_backward")

    def ray_query(self, rays, stream=None):
        """Closest hits against the tree of the last frame's broadphase and the
        current poses (see ray_query); not available on fused batched frames,
        which build no tree."""
        v = capi.BvhView()
        check(capi.lib().dyph_broadphase_bvh_view(self._bp, self.bodies.n, C.byref(v)))
        return ray_query(v, self.bodies, self.shapes, rays, stream)

    def contact_sensor(self, shape_idx: int):
        """ContactSensor(shape_idx).query over the last frame's contacts: (ab, p7)."""
        self.sync_lists()
        v = capi.Contacts()
        check(capi.lib().dyph_narrowphase_contacts(self._np, C.byref(v)))
        cs = ContactSensor(shape_idx)
        cs.query(v, self.bodies)
        return cs.rows()

    def bvh(self) -> dict:
        bp = Broadphase.__new__(Broadphase)
        bp.h = self._bp
        try:
            return bp.bvh(self.bodies.n)
        finally:
            bp.h = None

    def colors(self, n: int):
        """JP colours of the last frame's solve (UINT32_MAX on the sequential path) and the colour count."""
        self.sync_lists()
        out = np.empty(max(n, 1), np.uint32)
        nc = C.c_uint32()
        check(capi.lib().dyph_xpbd_download_colors(self._sv, None, out.ctypes.data_as(capi._up), n, C.byref(nc)))
        return out[:n], int(nc.value)

    def solver_stats(self) -> dict:
        """Path of the last frame's solve (0 sequential / none, 1 coloured attempt fell back to the
        sequential order, 2 coloured), its colour count and its Jones–Plassmann rounds."""
        v = [C.c_uint32() for _ in range(3)]
        check(capi.lib().dyph_xpbd_download_stats(self._sv, None, *[C.byref(x) for x in v]))
        return {"path": int(v[0].value), "colors": int(v[1].value), "rounds": int(v[2].value)}
