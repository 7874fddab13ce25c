"""Ray queries and the contact sensor.

CPU: the oracle's restatement (dyo_ray_query / dyo_contact_sensor) against
the reference's own ray_query / ContactSensor built in oracle/_ref, bit for
bit, and the reference's known answers (core/tests/ray_query_test.cpp,
bindings/python/tests/test_contact_sensor.py).
GPU: dyph_ray_query / dyph_contact_sensor_* against the oracle, bit for bit.
"""
import numpy as np
import pytest

from dyphur_b200 import scenes
from test_oracle_pins import _single_scene

UMAX = 0xFFFFFFFF
SPHERE, BOX = (1, 1.0, 1.0, 1.0), (0, 1.0, 1.0, 1.0)


def _ray(ox, oy, oz, dx, dy, dz, t_max=1e9):
    return [ox, oy, oz, dx, dy, dz, t_max]


# (name, shape, body positions, bounds, rays, expected (t, body) per ray)
# after ray_query_test.cpp:44-197.
RAY_KATS = [
    ("sphere_x", SPHERE, [[0, 0, 0], [0, 50, 0]], [-6, -6, -6, 56, 56, 56],
     [_ray(-5, 0, 0, 1, 0, 0), _ray(-5, 3, 0, 1, 0, 0)], [(4.0, 0), (None, UMAX)]),
    ("box_x", BOX, [[0, 0, 0], [0, 50, 0]], [-6, -6, -6, 56, 56, 56],
     [_ray(-5, 0, 0, 1, 0, 0), _ray(-5, 2, 0, 1, 0, 0)], [(4.0, 0), (None, UMAX)]),
    ("closest_of_two", SPHERE, [[0, 0, 0], [10, 0, 0]], [-6, -6, -6, 12, 6, 6],
     [_ray(-5, 0, 0, 1, 0, 0)], [(4.0, 0)]),
    ("t_max_caps", SPHERE, [[0, 0, 0], [50, 0, 0]], [-6, -6, -6, 56, 6, 6],
     [_ray(-5, 0, 0, 1, 0, 0, 2.0)], [(None, UMAX)]),
]


def _kat_scene(shape, pos, bounds):
    s = _single_scene([0] * len(pos), pos, [shape])
    s.bounds = np.array([bounds], np.float32)
    return s


def _check_kat(t, body, expect):
    for k, (et, eb) in enumerate(expect):
        assert int(body[k]) == eb, f"ray {k}: body {int(body[k])} != {eb}"
        if et is not None:
            assert abs(float(t[k]) - et) < 1e-3


def _random_rays(scene, n, seed):
    """Rays from outside each body's neighbourhood aimed near random bodies,
    plus axis-aligned rays (zero direction components) and capped t_max."""
    rng = np.random.default_rng(seed)
    lo, hi = scene.bounds[0, :3], scene.bounds[0, 3:]
    target = scene.pos[rng.integers(0, scene.n_bodies, n)] + rng.normal(0, 0.4, (n, 3))
    origin = rng.uniform(lo - 2, hi + 2, (n, 3))
    d = target - origin
    axis = rng.random(n) < 0.25
    k = rng.integers(0, 3, n)
    d[axis] = 0.0
    d[axis, k[axis]] = np.where(rng.random(axis.sum()) < 0.5, -1.0, 1.0)
    origin[axis] = target[axis] - 30.0 * d[axis]
    t_max = np.where(rng.random(n) < 0.2, rng.uniform(0.5, 40.0, n), 1e9)
    return np.concatenate([origin, d, t_max[:, None]], 1).astype(np.float32)


def _pile_after(oracle_mod, which, n, frames):
    s = scenes.random_pile(n, seed=7)
    w = oracle_mod.World(s, which)
    assert w.step(frames) == 0
    return s, w


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name,shape,pos,bounds,rays,expect", RAY_KATS, ids=[k[0] for k in RAY_KATS])
def test_oracle_ray_kats(oracle_mod, name, shape, pos, bounds, rays, expect):
    for which in ("oracle",) + (("ref",) if oracle_mod.ref_available() else ()):
        w = oracle_mod.World(_kat_scene(shape, pos, bounds), which)
        w.stage(oracle_mod.STAGE_BROADPHASE)
        t, body = w.ray_query(np.array(rays, np.float32))
        _check_kat(t, body, expect)


def test_oracle_ray_matches_reference(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference build absent")
    s, o = _pile_after(oracle_mod, "oracle", 2048, 40)
    _, r = _pile_after(oracle_mod, "ref", 2048, 40)
    rays = _random_rays(s, 4096, 11)
    to, bo = o.ray_query(rays)
    tr, br = r.ray_query(rays)
    assert np.array_equal(bo, br) and np.array_equal(bits(to), bits(tr))
    assert (bo != UMAX).sum() > 1000  # most rays hit something


def _sensor_shapes(scene, ab):
    """Shapes to subscribe to: the ground / box shapes of a shared-shape scene,
    or the shapes of the first bodies in contact, plus one no body has."""
    picks = set(scene.shape[ab[:40, 0]].tolist()) if len(ab) else set()
    return sorted(picks | {0, 1, int(scene.shape_type.shape[0]) + 5})


@pytest.mark.parametrize("which_scene", ["stress_blocks", "pile"])
def test_oracle_sensor_matches_reference(oracle_mod, which_scene):
    if not oracle_mod.ref_available():
        pytest.skip("reference build absent")
    if which_scene == "pile":
        s, o = _pile_after(oracle_mod, "oracle", 2048, 40)
        _, r = _pile_after(oracle_mod, "ref", 2048, 40)
    else:
        s = scenes.stress_blocks()
        o, r = oracle_mod.World(s, "oracle"), oracle_mod.World(s, "ref")
        assert o.step(60) == 0 and r.step(60) == 0
    all_ab, _ = o.contacts()
    matched = 0
    for shape_idx in _sensor_shapes(s, all_ab):
        (ao, po), (ar, pr) = o.contact_sensor(shape_idx), r.contact_sensor(shape_idx)
        assert np.array_equal(ao, ar) and np.array_equal(bits(po), bits(pr))
        matched += len(ao)
    assert matched > 20


def _two_spheres():
    """test_contact_sensor.py:14-50: radius-1 spheres at x = 0 and 1.5."""
    s = _single_scene([0, 0], [[0, 0, 0], [1.5, 0, 0]], [SPHERE])
    s.bounds = np.array([[-2, -2, -2, 4, 2, 2]], np.float32)
    return s


def test_oracle_sensor_two_spheres(oracle_mod):
    for which in ("oracle",) + (("ref",) if oracle_mod.ref_available() else ()):
        w = oracle_mod.World(_two_spheres(), which)
        for st in (oracle_mod.STAGE_BROADPHASE, oracle_mod.STAGE_NARROWPHASE):
            w.stage(st)
        ab, p7 = w.contact_sensor(0)
        assert len(ab) == 1 and p7[0, 6] > 0
        assert abs(np.linalg.norm(p7[0, 3:6]) - 1.0) < 1e-4
        assert len(w.contact_sensor(99)[0]) == 0


# ── GPU ──────────────────────────────────────────────────────────────────────


@pytest.fixture(scope="module")
def dev():
    from dyphur_b200 import device
    device.require_device()
    return device


def _device_stages(dev, scene, narrow=False):
    bodies, shapes = dev.DeviceBodies(scene), dev.DeviceShapes(scene)
    bp = dev.Broadphase(scene.n_bodies, scene.max_pairs)
    bp.build_and_query(bodies, shapes, scene.bounds[0])
    np_ = None
    if narrow:
        np_ = dev.Narrowphase(scene.max_contacts)
        np_.run(bp, bodies, shapes)
    return bodies, shapes, bp, np_


@pytest.mark.gpu
@pytest.mark.parametrize("name,shape,pos,bounds,rays,expect", RAY_KATS, ids=[k[0] for k in RAY_KATS])
def test_gpu_ray_kats(dev, oracle_mod, name, shape, pos, bounds, rays, expect):
    s = _kat_scene(shape, pos, bounds)
    bodies, shapes, bp, _ = _device_stages(dev, s)
    t, body = dev.ray_query(bp.bvh_view(s.n_bodies), bodies, shapes, np.array(rays, np.float32))
    t, body = t.cpu().numpy(), body.cpu().numpy().view(np.uint32)
    _check_kat(t, body, expect)
    o = oracle_mod.World(s)
    o.stage(oracle_mod.STAGE_BROADPHASE)
    to, bo = o.ray_query(np.array(rays, np.float32))
    assert np.array_equal(body, bo) and np.array_equal(bits(t), bits(to))


@pytest.mark.gpu
def test_gpu_ray_single_and_empty(dev, oracle_mod):
    """One body: no tree, the leaf test on body 0 (ray_query.cpp:162-166)."""
    s = _kat_scene(BOX, [[0, 0, 0]], [-6, -6, -6, 6, 6, 6])
    bodies, shapes, bp, _ = _device_stages(dev, s)
    rays = np.array([_ray(-5, 0.5, 0, 1, 0, 0), _ray(-5, 5, 0, 1, 0, 0)], np.float32)
    t, body = dev.ray_query(bp.bvh_view(1), bodies, shapes, rays)
    assert body.cpu().numpy().view(np.uint32).tolist() == [0, UMAX]
    assert abs(float(t[0]) - 4.0) < 1e-6
    t, body = dev.ray_query(bp.bvh_view(0), bodies, shapes, rays)  # empty tree: every ray misses
    assert body.cpu().numpy().view(np.uint32).tolist() == [UMAX, UMAX]
    assert np.array_equal(t.cpu().numpy(), rays[:, 6])


@pytest.mark.gpu
@pytest.mark.parametrize("n,frames", [(4096, 60), (65536, 30)])
def test_gpu_ray_random_pile(dev, oracle_mod, n, frames):
    which = "ref" if oracle_mod.ref_available() else "oracle"
    s, o = _pile_after(oracle_mod, which, n, frames)
    w = dev.World(s)
    w.step(frames)
    rays = _random_rays(s, 1 << 16, 5)
    t, body = w.ray_query(rays)
    to, bo = o.ray_query(rays)
    body = body.cpu().numpy().view(np.uint32)
    assert np.array_equal(body, bo) and np.array_equal(bits(t.cpu().numpy()), bits(to))
    assert (bo != UMAX).mean() > 0.3


@pytest.mark.gpu
def test_gpu_sensor_two_spheres(dev):
    s = _two_spheres()
    bodies, shapes, bp, np_ = _device_stages(dev, s, narrow=True)
    cs = dev.ContactSensor(0)
    assert cs.query(np_.contacts_view(), bodies) == 1 and cs.count() == 1 and cs.shape_idx() == 0
    ab, p7 = cs.rows()
    assert ab.tolist() == [[0, 1]] and p7[0, 6] > 0 and abs(np.linalg.norm(p7[0, 3:6]) - 1) < 1e-4
    assert dev.ContactSensor(99).query(np_.contacts_view(), bodies) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("which_scene", ["stress_blocks", "pile65k"])
def test_gpu_sensor_matches_oracle(dev, oracle_mod, which_scene):
    which = "ref" if oracle_mod.ref_available() else "oracle"
    if which_scene == "pile65k":
        s, o = _pile_after(oracle_mod, which, 65536, 60)
        frames = 60
    else:
        s, frames = scenes.stress_blocks(), 60
        o = oracle_mod.World(s, which)
        assert o.step(frames) == 0
    w = dev.World(s)
    w.step(frames)
    all_ab, _ = o.contacts()
    matched = 0
    for shape_idx in _sensor_shapes(s, all_ab):
        ab, p7 = w.contact_sensor(shape_idx)
        ao, po = o.contact_sensor(shape_idx)
        assert np.array_equal(ab, ao) and np.array_equal(bits(p7), bits(po)), f"shape {shape_idx}"
        matched += len(ab)
    assert matched > 20
