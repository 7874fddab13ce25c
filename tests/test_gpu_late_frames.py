"""Parity on the benchmarked configuration and the reference's own KAT scenes,
both through the CUDA path.

1. The large single-scene stress (65,536 bodies + ground, seed 2, 600 frames)
   is stepped on the GPU and by the reference's own sources built on the host
   (oracle/_ref, OpenMP on every host core; the C restatement when that build
   is absent). After 100, 200, 400 and 600 frames every body float, the pair
   list, the contact rows and the JP colours are compared bit for bit. The
   frames whose solve fell back to the sequential order are recorded and must
   include some: those are the frames where per-body list overflow, the
   per-thread item limit and the look-back order are exercised at scale.
2. The reference's KAT scenes (core/tests/narrowphase_test.cpp:217-343,
   broadphase_test.cpp:53-131, xpbd_solver_test.cpp:182-215 and 302-375) run
   through the CUDA stages and are checked against the published values and,
   bit for bit, against the oracle.
"""
import numpy as np
import pytest

from dyphur_b200 import scenes
from test_oracle_pins import NP_CASES, _single_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from dyphur_b200 import device
    device.require_device()
    return device


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_random_pile_65k_late_frames(dev, oracle_mod):
    s = scenes.random_pile(65536, seed=2)
    which = "ref" if oracle_mod.ref_available() else "oracle"
    o = oracle_mod.World(s, which)
    w = dev.World(s)
    fallback_frames, colored_frames = [], []
    frame = o_frame = 0
    for check_at in (100, 200, 400, 600):
        while frame < check_at:
            w.step(1)
            st = w.solver_stats()
            if st["path"] == 1:
                fallback_frames.append(frame)
            elif st["path"] == 2:
                colored_frames.append(frame)
            frame += 1
        assert o.step(check_at - o_frame, 0) == 0
        o_frame = check_at
        assert w.stats()["status"] == 0 and dev.device_error() == 0
        assert np.array_equal(bits(w.state()), bits(o.state())), f"state after {frame} frames"
        po, npo = o.pairs()
        assert np.array_equal(w.pairs(), po), f"pairs after {frame} frames"
        (ag, cg), (ao, co) = w.contacts(), o.contacts()
        assert np.array_equal(ag, ao), f"contact pairs after {frame} frames"
        assert np.array_equal(bits(cg), bits(co)), f"contact rows after {frame} frames"
        oc = o.colors()
        gc, ncol = w.colors(len(ao))
        if np.all(oc == 0xFFFFFFFF):
            assert ncol == 0, f"the reference fell back to the sequential order after {frame} frames"
        else:
            assert ncol > 0 and np.array_equal(gc, oc), f"JP colours after {frame} frames"
    assert w.hash() == o.hash()
    print(f"\n{which}: {len(fallback_frames)} fallback frames (first {fallback_frames[:8]}), "
          f"{len(colored_frames)} coloured frames")
    assert fallback_frames, "no frame took the sequential fallback"
    assert colored_frames, "no frame took the coloured path"


def _stages(dev, scene):
    bodies, shapes = dev.DeviceBodies(scene), dev.DeviceShapes(scene)
    bp = dev.Broadphase(scene.n_bodies, scene.max_pairs)
    bp.build_and_query(bodies, shapes, scene.bounds[0])
    return bodies, shapes, bp


def test_kat_broadphase_three_spheres(dev):
    """broadphase_test.cpp:53-87: exactly pair (0, 1)."""
    s = _single_scene([0, 0, 0], [[0, 0, 0], [1, 0, 0], [100, 0, 0]], [(1, 1.0, 0.5, 0.5)])
    s.bounds = np.array([[-2, -2, -2, 102, 2, 2]], np.float32)
    _, _, bp = _stages(dev, s)
    assert bp.download_count() == 1 and bp.pairs().tolist() == [[0, 1]]


def test_kat_broadphase_four_spheres(dev):
    """broadphase_test.cpp:90-131: all six a < b pairs, in ascending order."""
    s = _single_scene([0] * 4, [[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0], [0, 0, 0.5]], [(1, 1.0, 0.5, 0.5)])
    s.bounds = np.array([[-2, -2, -2, 2, 2, 2]], np.float32)
    _, _, bp = _stages(dev, s)
    assert bp.pairs().tolist() == [[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]]


@pytest.mark.parametrize("name,shape_of,pos,shapes,expect", NP_CASES, ids=[c[0] for c in NP_CASES])
def test_kat_narrowphase(dev, oracle_mod, name, shape_of, pos, shapes, expect):
    s = _single_scene(shape_of, pos, shapes)
    s.bounds = np.array([[-5, -5, -5, 5, 5, 5]], np.float32)
    bodies, shapes_d, bp = _stages(dev, s)
    npz = dev.Narrowphase(s.max_contacts)
    npz.run(bp, bodies, shapes_d)
    ab, p7 = npz.contacts()
    assert len(ab) == 1
    depth, nrm, pt = expect
    assert abs(p7[0, 6] - depth) < 1e-4
    assert np.allclose(p7[0, 3:6], nrm, atol=1e-4)
    for k, v in enumerate(pt):
        if v is not None:
            assert abs(p7[0, k] - v) < 1e-4
    o = oracle_mod.World(s)
    o.stage(oracle_mod.STAGE_BROADPHASE)
    o.stage(oracle_mod.STAGE_NARROWPHASE)
    ao, co = o.contacts()
    assert np.array_equal(ab, ao) and np.array_equal(bits(p7), bits(co))


def test_kat_solver_sphere_pair_separates(dev, oracle_mod):
    """xpbd_solver_test.cpp:182-215: one solver pass pushes two overlapping spheres apart."""
    s = _single_scene([0, 0], [[0, 0, 0], [0, 1.5, 0]], [(1, 1.0, 0.5, 0.5)])
    s.bounds = np.array([[-5, -5, -5, 5, 5, 5]], np.float32)
    s.n_iters = 1
    bodies, shapes_d, bp = _stages(dev, s)
    npz = dev.Narrowphase(s.max_contacts)
    npz.run(bp, bodies, shapes_d)
    sv = dev.XpbdSolver(1, s.max_contacts, s.n_bodies, s.friction)
    sv.solve(npz.contacts_view(), bodies, s.dt)
    y = bodies.state()[1]
    assert y[1] - y[0] >= 2.0 - 1e-3
    o = oracle_mod.World(s)
    for st in (oracle_mod.STAGE_BROADPHASE, oracle_mod.STAGE_NARROWPHASE, oracle_mod.STAGE_SOLVE):
        o.stage(st)
    assert np.array_equal(bits(bodies.state()), bits(o.state()))


def test_kat_colored_equals_sequential_on_independent_pairs(dev, oracle_mod):
    """xpbd_solver_test.cpp:302-375: 300 disjoint sphere pairs (above the 256-contact
    threshold, so the reference mode colours) give the same bits as the sequential order."""
    n_pairs = 300
    pos = []
    for k in range(n_pairs):
        pos += [[0, 10.0 * k, 0], [0, 10.0 * k + 0.8, 0]]
    s = _single_scene([0] * (2 * n_pairs), pos, [(1, 0.5, 0.5, 0.5)])
    s.bounds = np.array([[-10, -10, -10, 10, 3010, 10]], np.float32)
    s.max_pairs, s.max_contacts = 4096, 4096
    out = {}
    for mode in (0, 1, 2, 3):
        bodies, shapes_d, bp = _stages(dev, s)
        npz = dev.Narrowphase(s.max_contacts)
        npz.run(bp, bodies, shapes_d)
        assert npz.download_count()[0] == n_pairs
        sv = dev.XpbdSolver(s.n_iters, s.max_contacts, s.n_bodies, s.friction)
        sv.set_mode(mode)
        sv.solve(npz.contacts_view(), bodies, s.dt)
        if mode in (0, 2):
            assert sv.colors(n_pairs)[1] > 0, "the coloured path ran"
        out[mode] = bits(bodies.state())
    for mode in (0, 2, 3):
        assert np.array_equal(out[mode], out[1]), mode
    o = oracle_mod.World(s)
    for st in (oracle_mod.STAGE_BROADPHASE, oracle_mod.STAGE_NARROWPHASE, oracle_mod.STAGE_SOLVE):
        o.stage(st, 0)
    assert np.array_equal(out[0], bits(o.state()))
