"""The dyphur_py extension module: the reference's Python surface
(bindings/python/dyphur_py.cpp:29-163) plus World, ray_query and rollout.

The GPU half ports bindings/python/tests/test_contact_sensor.py (two touching
spheres, one contact, zero-copy numpy views) and checks the module's frame
step and rollout against the oracle and the ctypes layer.
"""
import numpy as np
import pytest

import dyphur_b200
from dyphur_b200 import scenes

# Classes and methods the reference binds (dyphur_py.cpp:29-163).
REFERENCE_SURFACE = {
    "Device": ["default_cpu", "make_stream"],
    "Stream": ["wait"],
    "AABB": ["min_x", "min_y", "min_z", "max_x", "max_y", "max_z"],
    "ShapeType": ["Box", "Sphere"],
    "ShapeParams": ["type", "half_x", "half_y", "half_z"],
    "ShapeStore": ["add", "upload", "count", "view"],
    "ShapeView": [],
    "BodyParams": ["set_position", "set_velocity", "mass", "shape_handle", "flags"],
    "BodyView": [],
    "BodyStore": ["add", "upload", "count", "view", "body_shapes"],
    "Broadphase": ["build_and_query", "download_count"],
    "Narrowphase": ["run", "download_count"],
    "ContactSensor": ["query", "count", "shape_idx", "body_a", "body_b", "pos_x", "pos_y", "pos_z", "norm_x",
                      "norm_y", "norm_z", "depth"],
}


@pytest.fixture(scope="module")
def dp():
    return dyphur_b200.import_dyphur_py()


def test_module_has_reference_surface(dp):
    for cls, members in REFERENCE_SURFACE.items():
        c = getattr(dp, cls)
        for m in members:
            assert hasattr(c, m), f"{cls}.{m}"
    assert hasattr(dp, "Box") and hasattr(dp, "Sphere")  # export_values
    for extra in ("World", "ray_query", "rollout", "integrate", "XpbdSolver", "FusedConfig"):
        assert hasattr(dp, extra)


# ── GPU ──────────────────────────────────────────────────────────────────────


@pytest.fixture(scope="module")
def two_sphere_scene(dp):
    """test_contact_sensor.py:14-50, on the default device (there is no CPU one)."""
    from dyphur_b200 import device
    device.require_device()
    dev = dp.Device.default_cpu()
    s = dev.make_stream()
    ss = dp.ShapeStore(s, 4)
    sp = dp.ShapeParams()
    sp.type = dp.ShapeType.Sphere
    sp.half_x = 1.0
    ss.add(sp)
    ss.upload()
    bs = dp.BodyStore(s, 4)
    p = dp.BodyParams()
    p.mass = 1.0
    p.shape_handle = 0
    p.set_position(0.0, 0.0, 0.0)
    bs.add(p)
    p.set_position(1.5, 0.0, 0.0)
    bs.add(p)
    bs.upload()
    s.wait()
    scene = dp.AABB(-2.0, -2.0, -2.0, 4.0, 2.0, 2.0)
    bp = dp.Broadphase(s, 4, 32)
    bp.build_and_query(s, bs.view(), ss.view(), scene)
    s.wait()
    n_pairs = bp.download_count(s)
    np_ = dp.Narrowphase(s, 32)
    np_.run(s, bp, n_pairs, bs.view(), ss.view())
    s.wait()
    return s, bp, np_, bs, ss, n_pairs


@pytest.mark.gpu
def test_broadphase_finds_pair(two_sphere_scene):
    assert two_sphere_scene[5] == 1


@pytest.mark.gpu
def test_narrowphase_finds_contact(two_sphere_scene):
    s, _, np_, _, _, _ = two_sphere_scene
    assert np_.download_count(s) == 1


@pytest.mark.gpu
def test_contact_sensor_count_depth_normal(dp, two_sphere_scene):
    s, _, np_, bs, _, _ = two_sphere_scene
    sensor = dp.ContactSensor(0)
    assert sensor.query(s, np_, bs.body_shapes()) == 1 and sensor.count() == 1
    depth = sensor.depth()
    assert len(depth) == 1 and float(depth[0]) > 0.0
    mag = float(np.sqrt(sensor.norm_x()[0] ** 2 + sensor.norm_y()[0] ** 2 + sensor.norm_z()[0] ** 2))
    assert abs(mag - 1.0) < 1e-4
    assert sensor.body_a().tolist() == [0] and sensor.body_b().tolist() == [1]


@pytest.mark.gpu
def test_contact_sensor_numpy_zero_copy(dp, two_sphere_scene):
    s, _, np_, bs, _, _ = two_sphere_scene
    sensor = dp.ContactSensor(0)
    sensor.query(s, np_, bs.body_shapes())
    assert not np.asarray(sensor.depth()).flags["OWNDATA"]
    assert not np.asarray(sensor.body_a()).flags["OWNDATA"]


@pytest.mark.gpu
def test_contact_sensor_no_hit_wrong_shape(dp, two_sphere_scene):
    s, _, np_, bs, _, _ = two_sphere_scene
    assert dp.ContactSensor(99).query(s, np_, bs.body_shapes()) == 0


@pytest.mark.gpu
def test_ray_query_kat(dp, two_sphere_scene):
    """ray_query_test.cpp:44-80 style: a ray along +x enters sphere 0 at x = -1."""
    s, bp, _, bs, ss, _ = two_sphere_scene
    rays = np.array([[-5, 0, 0, 1, 0, 0, 1e9], [-5, 3, 0, 1, 0, 0, 1e9], [-5, 0, 0, 1, 0, 0, 2.0]], np.float32)
    t, body = dp.ray_query(s, bp.bvh_view(bs.count()), bs.view(), ss.view(), rays)
    assert body.tolist() == [0, 0xFFFFFFFF, 0xFFFFFFFF]
    assert abs(float(t[0]) - 4.0) < 1e-3


def _stores(dp, s, scene):
    ss = dp.ShapeStore(s, int(scene.shape_type.shape[0]))
    for k in range(int(scene.shape_type.shape[0])):
        sp = dp.ShapeParams()
        sp.type = dp.ShapeType.Sphere if scene.shape_type[k] == 1 else dp.ShapeType.Box
        sp.half_x, sp.half_y, sp.half_z = (float(x) for x in scene.shape_half[k])
        ss.add(sp)
    ss.upload()
    bs = dp.BodyStore(s, scene.n_bodies)
    for i in range(scene.n_bodies):
        p = dp.BodyParams()
        p.set_position(*(float(x) for x in scene.pos[i]))
        p.set_rotation(*(float(x) for x in scene.rot[i]))
        p.set_velocity(*(float(x) for x in scene.vel[i]))
        p.set_angular_velocity(*(float(x) for x in scene.ang[i]))
        p.set_inertia([float(x) for x in scene.inertia[i]])
        p.mass = float(scene.mass[i])
        p.shape_handle = int(scene.shape[i])
        p.flags = int(scene.flags[i])
        bs.add(p)
    bs.upload()
    return ss, bs


def _params(dp, scene):
    ip = dp.IntegratorParams()
    ip.set_gravity(*scene.gravity)
    ip.dt = scene.dt
    ip.n_substeps = scene.n_substeps
    return ip


@pytest.mark.gpu
def test_world_step_matches_oracle(dp, oracle_mod):
    from dyphur_b200 import device
    device.require_device()
    scene = scenes.stress_blocks()
    s = dp.Device.default_gpu().make_stream()
    ss, bs = _stores(dp, s, scene)
    b = scene.bounds[0]
    w = dp.World(s, bs, ss, dp.AABB(*(float(x) for x in b)), _params(dp, scene), scene.max_pairs,
                 scene.max_contacts, scene.n_iters, scene.friction)
    w.step(s, 40)
    s.wait()
    o = oracle_mod.World(scene)
    assert o.step(40) == 0
    assert np.array_equal(bs.state().view(np.uint32), o.state().view(np.uint32))
    assert w.hash(s) == o.hash()


@pytest.mark.gpu
def test_rollout_through_module_matches_ctypes_world(dp):
    """dp.rollout (the autograd function over dp.World) gives the same final
    state and gradients, bit for bit, as the same rollout over device.World."""
    import torch

    from dyphur_b200 import autograd, device
    device.require_device()
    scene = scenes.push(4)
    n = scene.n_bodies
    s = dp.Device.default_gpu().make_stream()
    ss, bs = _stores(dp, s, scene)
    w = dp.World(s, bs, ss, dp.AABB(*(float(x) for x in scene.bounds[0])), _params(dp, scene),
                 48 * n + 64 * scene.n_scenes, 16 * n + 64 * scene.n_scenes, scene.n_iters, scene.friction,
                 dp.SolverMode.Sequential)
    w.set_scenes([int(x) for x in scene.body_offset], [dp.AABB(*(float(x) for x in b)) for b in scene.bounds])
    s.wait()
    cfg = w.autotune(s, 4)  # the configuration changes no frame
    assert cfg.blocks >= 1 and cfg.warp_scenes + cfg.half_scenes + cfg.block_scenes == scene.n_scenes
    wc = device.World(scene, mode=1)
    target = torch.from_numpy(scene.targets).cuda()
    results = []
    for world, roll in ((w, dp.rollout), (wc, autograd.rollout)):
        rows = torch.as_tensor(world.device_rows(), device="cuda") if world is w else world.device_rows()
        init = torch.as_tensor(world.initial_rows(), device="cuda") if world is w else world.initial_rows()
        vel = init[7:10, :n].T.clone().requires_grad_(True)
        ang = init[10:13, :n].T.clone().requires_grad_(True)
        im = rows[13, :n].clone().requires_grad_(True)
        final = roll(world, vel, ang, im, 40, 10)
        loss = ((final[:3].T - target) ** 2).sum()
        loss.backward()
        torch.cuda.synchronize()
        results.append((final.detach().cpu(), vel.grad.cpu(), ang.grad.cpu(), im.grad.cpu()))
    for a, b in zip(*results):
        assert torch.equal(a, b)
    assert results[0][1].abs().sum() > 0


@pytest.mark.gpu
def test_backward_after_the_scenes_change(dp):
    """The adjoint's record sets are sized by the scenes' slots: after
    set_scenes changes them, a backward pass equals, bit for bit, that of a
    world set up with the new scenes from the start."""
    import torch

    from dyphur_b200 import device
    device.require_device()
    scene = scenes.push(4)
    n = scene.n_bodies
    off = [int(x) for x in scene.body_offset]
    merged = [off[0], off[2], off[4]]  # two scenes of two pushes each

    def aabb(lo, hi):
        b = np.concatenate([scene.bounds[lo:hi, :3].min(0), scene.bounds[lo:hi, 3:].max(0)])
        return dp.AABB(*(float(x) for x in b))

    def world(s):
        ss, bs = _stores(dp, s, scene)
        w = dp.World(s, bs, ss, aabb(0, 4), _params(dp, scene), 48 * n + 256, 16 * n + 256, scene.n_iters,
                     scene.friction, dp.SolverMode.Sequential)
        return w, (ss, bs)

    def grads(w):
        rows = torch.as_tensor(w.device_rows(), device="cuda")
        init = torch.as_tensor(w.initial_rows(), device="cuda")
        vel = init[7:10, :n].T.clone().requires_grad_(True)
        ang = init[10:13, :n].T.clone().requires_grad_(True)
        im = rows[13, :n].clone().requires_grad_(True)
        final = dp.rollout(w, vel, ang, im, 12, 4)
        (final[:3] ** 2).sum().backward()
        torch.cuda.synchronize()
        return [t.grad.cpu().numpy() for t in (vel, ang, im)]

    s = dp.Device.default_gpu().make_stream()
    w, keep = world(s)
    w.set_scenes(off, [aabb(i, i + 1) for i in range(4)])
    s.wait()
    grads(w)
    w.set_scenes(merged, [aabb(0, 2), aabb(2, 4)])
    s.wait()
    got = grads(w)
    w2, keep2 = world(s)
    w2.set_scenes(merged, [aabb(0, 2), aabb(2, 4)])
    s.wait()
    want = grads(w2)
    assert np.abs(want[0]).sum() > 0
    for a, b in zip(got, want):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
