"""ctypes bindings of the C ABI declared in ``include/dyphur_b200.h``."""
from __future__ import annotations

import ctypes as C

from ._lib import load_library

OK, ERR_INVALID, ERR_CUDA, ERR_PAIR_OVERFLOW, ERR_CONTACT_OVERFLOW, ERR_TIMEOUT, ERR_NO_DEVICE, ERR_NOMEM, \
    ERR_NOT_FINITE, ERR_TOO_LARGE, ERR_UNSUPPORTED = range(11)
SORT_NOALLOC_MAX_KEYS = 262144
SOLVER_REFERENCE, SOLVER_SEQUENTIAL, SOLVER_COLORED, SOLVER_REFERENCE_ROUNDS = 0, 1, 2, 3

_fp = C.POINTER(C.c_float)
_up = C.POINTER(C.c_uint32)


class Bodies(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in (
        "pos_x", "pos_y", "pos_z", "rot_w", "rot_x", "rot_y", "rot_z", "vel_x", "vel_y", "vel_z",
        "ang_x", "ang_y", "ang_z", "inv_mass", "iI_xx", "iI_yy", "iI_zz", "iI_xy", "iI_xz", "iI_yz",
        "shape", "flags")] + [("n", C.c_uint32)]


class Shapes(C.Structure):
    _fields_ = [("type", C.c_void_p), ("half_x", C.c_void_p), ("half_y", C.c_void_p), ("half_z", C.c_void_p),
                ("ext_id", C.c_void_p), ("n", C.c_uint32)]


class Contacts(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("body_a", "body_b", "pos_x", "pos_y", "pos_z", "norm_x", "norm_y",
                                          "norm_z", "depth", "n")] + [("capacity", C.c_uint32)]


class FusedConfig(C.Structure):
    _fields_ = [("smem_bytes", C.c_uint32), ("teams", C.c_uint32), ("warp_scenes", C.c_uint32),
                ("half_scenes", C.c_uint32), ("block_scenes", C.c_uint32), ("blocks", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("register_blocks", C.c_uint32), ("ms_per_frame", C.c_float), ("candidates", C.c_uint32)]


class AABB(C.Structure):
    _fields_ = [(f, C.c_float) for f in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")]


class BvhView(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("left", "right", "parent", "root", "sorted_idx", "aabb",
                                          "sorted_keys")] + [("n", C.c_uint32)]


class IntegratorParams(C.Structure):
    _fields_ = [("gravity", C.c_float * 3), ("dt", C.c_float), ("n_substeps", C.c_int32)]


class WorldDesc(C.Structure):
    _fields_ = [("bodies", Bodies), ("shapes", Shapes), ("scene_bounds", AABB), ("integrator", IntegratorParams),
                ("max_pairs", C.c_uint32), ("max_contacts", C.c_uint32), ("n_iters", C.c_int32),
                ("friction", C.c_float), ("mode", C.c_int)]


_vp = C.c_void_p
_st = C.c_int
_PROTOS = {
    "dyph_status_string": (C.c_char_p, [C.c_int]),
    "dyph_last_cuda_error": (C.c_char_p, []),
    "dyph_device_check": (_st, []),
    "dyph_download_device_error": (_st, [_vp, _up]),
    "dyph_download_device_error_site": (_st, [_vp, _up, _up]),
    "dyph_integrate": (_st, [C.POINTER(Bodies), C.POINTER(IntegratorParams), _vp]),
    "dyph_sort_workspace_bytes": (C.c_size_t, [C.c_size_t]),
    "dyph_sort_by_key_u64_u32": (_st, [_vp, _vp, C.c_size_t, _vp, C.c_size_t, _vp]),
    "dyph_sort_by_key_u64_u32_noalloc": (_st, [_vp, _vp, C.c_size_t, _vp]),
    "dyph_broadphase_set_scenes": (_st, [_vp, C.c_uint32, _vp, _vp]),
    "dyph_world_set_scenes": (_st, [_vp, C.c_uint32, _vp, _vp]),
    "dyph_world_scene_hashes": (_st, [_vp, _vp, _vp, C.c_uint32]),
    "dyph_sort_u64": (_st, [_vp, C.c_size_t, _vp, C.c_size_t, _vp]),
    "dyph_sort_by_key_u32_u32": (_st, [_vp, _vp, C.c_size_t, C.c_int, _vp, C.c_size_t, _vp]),
    "dyph_broadphase_create": (_st, [C.c_uint32, C.c_uint32, C.POINTER(_vp)]),
    "dyph_broadphase_destroy": (None, [_vp]),
    "dyph_broadphase_build_and_query": (_st, [_vp, C.POINTER(Bodies), C.POINTER(Shapes), C.POINTER(AABB), _vp]),
    "dyph_broadphase_sort_pairs": (_st, [_vp, C.c_uint32, _vp]),
    "dyph_broadphase_download_count": (_st, [_vp, _vp, _up]),
    "dyph_broadphase_pairs": (_vp, [_vp]),
    "dyph_broadphase_count_ptr": (_vp, [_vp]),
    "dyph_broadphase_max_pairs": (C.c_uint32, [_vp]),
    "dyph_broadphase_bvh_view": (_st, [_vp, C.c_uint32, C.POINTER(BvhView)]),
    "dyph_narrowphase_create": (_st, [C.c_uint32, C.POINTER(_vp)]),
    "dyph_narrowphase_destroy": (None, [_vp]),
    "dyph_narrowphase_run": (_st, [_vp, _vp, _vp, C.POINTER(Bodies), C.POINTER(Shapes), _vp]),
    "dyph_narrowphase_run_host_count": (_st, [_vp, _vp, C.c_uint32, C.POINTER(Bodies), C.POINTER(Shapes), _vp]),
    "dyph_narrowphase_contacts": (_st, [_vp, C.POINTER(Contacts)]),
    "dyph_narrowphase_download_count": (_st, [_vp, _vp, _up, _up]),
    "dyph_set_spin_limit": (_st, [C.c_uint32]),
    "dyph_wait_selftest": (_st, [C.c_int, _vp]),
    "dyph_bodies_check_finite": (_st, [C.POINTER(Bodies), _vp, _up]),
    "dyph_world_check_finite": (_st, [_vp, _vp, _up]),
    "dyph_world_fused_config": (_st, [_vp, C.POINTER(FusedConfig)]),
    "dyph_world_set_fused_config": (_st, [_vp, C.c_uint32, C.c_uint32, C.c_uint32]),
    "dyph_world_autotune": (_st, [_vp, C.c_int32, _vp, C.POINTER(FusedConfig)]),
    "dyph_world_adjoint_config": (_st, [_vp, C.POINTER(FusedConfig)]),
    "dyph_world_set_adjoint_config": (_st, [_vp, C.c_uint32, C.c_uint32]),
    "dyph_ray_query": (_st, [C.POINTER(BvhView), C.POINTER(Bodies), C.POINTER(Shapes), _vp, _vp, C.c_uint32, _vp]),
    "dyph_contact_sensor_create": (_st, [C.c_uint32, C.POINTER(_vp)]),
    "dyph_contact_sensor_destroy": (None, [_vp]),
    "dyph_contact_sensor_filter": (_st, [_vp, C.POINTER(Contacts), _vp, C.c_uint32, _vp]),
    "dyph_contact_sensor_query": (_st, [_vp, C.POINTER(Contacts), _vp, C.c_uint32, _vp, _up]),
    "dyph_contact_sensor_count": (C.c_uint32, [_vp]),
    "dyph_contact_sensor_shape_idx": (C.c_uint32, [_vp]),
    "dyph_contact_sensor_host_view": (_st, [_vp, C.POINTER(Contacts)]),
    "dyph_contact_sensor_device_view": (_st, [_vp, C.POINTER(Contacts)]),
    "dyph_xpbd_create": (_st, [C.c_int32, C.c_uint32, C.c_uint32, C.c_float, C.POINTER(_vp)]),
    "dyph_xpbd_destroy": (None, [_vp]),
    "dyph_xpbd_set_mode": (_st, [_vp, C.c_int]),
    "dyph_xpbd_solve": (_st, [_vp, C.POINTER(Contacts), C.POINTER(Bodies), C.c_float, _vp]),
    "dyph_xpbd_download_colors": (_st, [_vp, _vp, _up, C.c_uint32, _up]),
    "dyph_xpbd_download_stats": (_st, [_vp, _vp, _up, _up, _up]),
    "dyph_xpbd_download_phase_ns": (_st, [_vp, _vp, _vp]),
    "dyph_fnv1a64_state": (_st, [C.POINTER(Bodies), _vp, _vp]),
    "dyph_world_create": (_st, [C.POINTER(WorldDesc), _vp, C.POINTER(_vp)]),
    "dyph_world_destroy": (None, [_vp]),
    "dyph_world_step": (_st, [_vp, C.c_int32, _vp]),
    "dyph_world_download_stats": (_st, [_vp, _vp, _up, _up, _up, _up, _up]),
    "dyph_world_broadphase": (_st, [_vp, C.POINTER(_vp)]),
    "dyph_world_narrowphase": (_st, [_vp, C.POINTER(_vp)]),
    "dyph_world_solver": (_st, [_vp, C.POINTER(_vp)]),
    "dyph_world_capture_episode": (_st, [_vp, C.c_int32, C.c_int32, C.POINTER(_vp), C.POINTER(_vp)]),
    "dyph_world_run_episode": (_st, [_vp, _vp]),
    "dyph_world_download_history": (_st, [_vp, _vp, _vp, _vp, C.c_uint32, _up]),
    "dyph_world_set_trajectory": (_st, [_vp, _vp, C.c_uint32, C.c_uint32]),
    "dyph_world_sync_lists": (_st, [_vp, _vp]),
    "dyph_world_rollout": (_st, [_vp, C.c_int32, C.c_int32, _vp, _vp]),
    "dyph_world_rollout_backward": (_st, [_vp, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp]),
    "dyph_world_set_phase_timing": (_st, [_vp, C.c_int]),
    "dyph_world_download_phase_ns": (_st, [_vp, _vp, _vp, C.c_uint32]),
    "dyph_event_create": (_st, [C.POINTER(_vp)]),
    "dyph_event_destroy": (None, [_vp]),
    "dyph_event_record": (_st, [_vp, _vp]),
    "dyph_event_elapsed_ms": (_st, [_vp, _vp, C.POINTER(C.c_float)]),
    "dyph_copy_to_host": (_st, [_vp, _vp, C.c_size_t, _vp]),
    "dyph_copy_to_device": (_st, [_vp, _vp, C.c_size_t, _vp]),
    "dyph_pack_bodies": (None, [C.c_uint32] + [_vp] * 11),
}

# Every symbol the header declares (checked by the CPU suite).
HEADER_SYMBOLS = tuple(_PROTOS)

_lib = None


def lib():
    global _lib
    if _lib is None:
        L = load_library()
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class DyphError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        msg = lib().dyph_status_string(status).decode()
        if status == ERR_CUDA:
            msg += ": " + lib().dyph_last_cuda_error().decode()
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")
        self.status = status


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise DyphError(status, what)
