"""Error paths, exercised without a GPU fault.

- Non-finite state: NaN / Inf written into the body state on the host is
  reported by dyph_bodies_check_finite / dyph_world_check_finite with the
  first bad body (nothing is stepped on it).
- Contact overflow: a world whose contact capacity is far below the scene's
  contact count keeps the ordered prefix, reports DYPH_ERR_CONTACT_OVERFLOW
  and still equals the oracle run with the same capacity, bit for bit.
- Timeouts: with a small spin limit, a look-back whose predecessor never
  publishes and a grid barrier whose second block never arrives give up,
  report DYPH_ERR_TIMEOUT with their site, and the context stays usable.
- Host-side argument checks that need no device.
"""
import ctypes as C

import numpy as np
import pytest

from dyphur_b200 import capi, scenes


def test_host_argument_checks():
    L = capi.lib()
    assert L.dyph_ray_query(None, None, None, None, None, 0, None) == capi.OK  # nothing to do
    assert L.dyph_ray_query(None, None, None, None, None, 4, None) == capi.ERR_INVALID
    assert L.dyph_wait_selftest(2, None) == capi.ERR_INVALID
    assert L.dyph_bodies_check_finite(None, None, None) == capi.ERR_INVALID
    assert L.dyph_world_check_finite(None, None, None) == capi.ERR_INVALID
    assert L.dyph_contact_sensor_filter(None, None, None, 0, None) == capi.ERR_INVALID
    assert L.dyph_contact_sensor_count(None) == 0
    assert L.dyph_world_adjoint_config(None, None) == capi.ERR_INVALID
    assert L.dyph_world_set_adjoint_config(None, 0, 1) == capi.ERR_INVALID
    assert L.dyph_world_set_fused_config(None, 0, 1, 0) == capi.ERR_INVALID
    assert L.dyph_world_rollout_backward(None, 1, 1, None, None, None, None, None) == capi.ERR_INVALID
    for code in range(11):
        assert capi.lib().dyph_status_string(code) not in (None, b"unknown status")


@pytest.fixture(scope="module")
def dev():
    from dyphur_b200 import device
    device.require_device()
    return device


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.gpu
def test_not_finite_reported(dev):
    s = scenes.stress_blocks()
    w = dev.World(s)
    w.step(5)
    first = C.c_uint32()
    assert capi.lib().dyph_world_check_finite(w.h, None, C.byref(first)) == capi.OK
    assert first.value == 0xFFFFFFFF
    st = w.state()
    good = st.copy()
    st[8, 17] = np.nan       # vel_y of body 17
    st[4, 300] = np.inf      # rot_x of body 300
    w.bodies.set_state(st)
    assert capi.lib().dyph_world_check_finite(w.h, None, C.byref(first)) == capi.ERR_NOT_FINITE
    assert first.value == 17
    st[8, 17] = good[8, 17]
    w.bodies.set_state(st)
    assert dev.check_finite(w.bodies) == (capi.ERR_NOT_FINITE, 300)
    w.bodies.set_state(good)
    assert dev.check_finite(w.bodies) == (capi.OK, 0xFFFFFFFF)
    assert dev.device_error() == 0


@pytest.mark.gpu
def test_contact_overflow_keeps_ordered_prefix(dev, oracle_mod):
    s = scenes.stress_blocks()
    cap = 256
    w = dev.World(s, mode=capi.SOLVER_SEQUENTIAL, max_contacts=cap)
    o = oracle_mod.World(s, max_contacts=cap)
    overflowed = 0
    for f in range(90):
        w.step(1)
        for st in (oracle_mod.STAGE_INTEGRATE, oracle_mod.STAGE_BROADPHASE, oracle_mod.STAGE_NARROWPHASE,
                   oracle_mod.STAGE_SOLVE):
            rc = o.stage(st, oracle_mod.SOLVER_SERIAL)
            if st == oracle_mod.STAGE_NARROWPHASE and rc == -3:
                overflowed += 1
            else:
                assert rc == 0
    assert overflowed > 10, "the scene never exceeded the contact capacity"
    stats = w.stats()
    assert stats["status"] == capi.ERR_CONTACT_OVERFLOW and stats["peak_contacts"] > cap
    assert np.array_equal(bits(w.state()), bits(o.state()))
    (ag, cg), (ao, co) = w.contacts(), o.contacts()
    assert len(ag) == cap and np.array_equal(ag, ao) and np.array_equal(bits(cg), bits(co))
    assert dev.device_error() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("which", [1, 3])
def test_bounded_wait_times_out_and_context_survives(dev, oracle_mod, which):
    assert dev.device_error() == 0
    dev.set_spin_limit(4096)
    try:
        dev.wait_selftest(which)
        assert dev.device_error_site() == (capi.ERR_TIMEOUT, which)
    finally:
        dev.set_spin_limit(0)
    # the context still steps a world bit-exactly
    s = scenes.determinism((4, 4, 4))
    w = dev.World(s)
    w.step(20)
    o = oracle_mod.World(s)
    assert o.step(20) == 0
    assert np.array_equal(bits(w.state()), bits(o.state()))
    assert dev.device_error_site() == (0, 0)
