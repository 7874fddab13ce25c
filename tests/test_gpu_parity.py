"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Integer / index outputs (Morton keys, BVH arrays, pair lists, contact pairs,
colours) and every float of the body state are compared bit for bit: the
kernels are built with --fmad=false and IEEE division / sqrt, so the
reference's float path is reproduced exactly (tolerance 0 ULP).
"""
import numpy as np
import pytest

from dyphur_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from dyphur_b200 import device
    device.require_device()
    return device


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def stage_parity(dev, oracle_mod, scene, frame, mode=0):
    """Advance the oracle to `frame`, then run each stage of the next frame on
    both sides from the same input state and compare every output."""
    o = oracle_mod.World(scene)
    assert o.step(frame, mode) == 0
    s0 = o.state()
    bodies = dev.DeviceBodies(scene)
    shapes = dev.DeviceShapes(scene)
    im_o, ii_o = o.inv()
    im_g, ii_g = bodies.inv()
    assert np.array_equal(bits(im_o), bits(im_g)) and np.array_equal(bits(ii_o), bits(ii_g))
    bodies.set_state(s0)
    # integrate
    o.stage(oracle_mod.STAGE_INTEGRATE)
    dev.integrate(bodies, scene.gravity, scene.dt, scene.n_substeps)
    assert np.array_equal(bits(o.state()), bits(bodies.state())), "integrate"
    # broadphase
    o.stage(oracle_mod.STAGE_BROADPHASE)
    bp = dev.Broadphase(scene.n_bodies, scene.max_pairs)
    bp.build_and_query(bodies, shapes, scene.bounds[0])
    po, npo = o.pairs()
    assert bp.download_count() == npo
    assert np.array_equal(bp.pairs(), po), "pairs"
    if scene.n_bodies >= 2:
        bo, bg = o.bvh(), bp.bvh(scene.n_bodies)
        for k in ("keys", "sorted_idx", "left", "right", "parent", "aabb"):
            assert np.array_equal(bo[k], bg[k]), k
    # narrowphase
    o.stage(oracle_mod.STAGE_NARROWPHASE)
    npz = dev.Narrowphase(scene.max_contacts)
    npz.run(bp, bodies, shapes)
    ao, co = o.contacts()
    ag, cg = npz.contacts()
    assert np.array_equal(ao, ag), "contact pairs"
    assert np.array_equal(bits(co), bits(cg)), "contact geometry"
    # solve
    o.stage(oracle_mod.STAGE_SOLVE, mode)
    sv = dev.XpbdSolver(scene.n_iters, scene.max_contacts, scene.n_bodies, scene.friction)
    sv.set_mode(mode)
    sv.solve(npz.contacts_view(), bodies, scene.dt)
    assert np.array_equal(bits(o.state()), bits(bodies.state())), "solve"
    if mode == 0 and len(ao) > 256:
        cols, ncol = sv.colors(len(ao))
        oc = o.colors()
        if np.all(oc == 0xFFFFFFFF):  # the reference fell back to the sequential order
            assert ncol == 0, "sequential fallback"
        else:
            assert ncol > 0 and np.array_equal(cols, oc), "JP colours"
    assert dev.device_error() == 0


@pytest.mark.parametrize("frame", [0, 22, 40, 90, 200])
def test_stage_parity_blocks(dev, oracle_mod, frame):
    stage_parity(dev, oracle_mod, scenes.stress_blocks(), frame)


@pytest.mark.parametrize("frame", [30, 120])
def test_stage_parity_blocks_sequential(dev, oracle_mod, frame):
    stage_parity(dev, oracle_mod, scenes.stress_blocks(), frame, mode=1)


@pytest.mark.parametrize("frame", [0, 2])
@pytest.mark.parametrize("mode", [0, 1])
def test_stage_parity_random_pile_65k(dev, oracle_mod, frame, mode):
    """Mode 1 here runs the sequential order on the dataflow kernel (> 2048 contacts)."""
    stage_parity(dev, oracle_mod, scenes.random_pile(65536), frame, mode=mode)


def test_world_determinism_golden(dev):
    """The reference's 8-box / 20-frame sim hash (core/tests/sim_determinism_test.cpp:224)."""
    w = dev.World(scenes.determinism())
    w.step(20)
    assert w.hash() == 0xcbcd209c3665c818


@pytest.mark.parametrize("mode", [0, 1, 3])
def test_world_blocks_300_frames(dev, oracle_mod, mode):
    """Modes 0 (reference: dataflow colouring above 256 contacts), 1 (sequential)
    and 3 (round-synchronous colouring, checked against the reference mode)."""
    s = scenes.stress_blocks()
    o = oracle_mod.World(s)
    assert o.step(300, 0 if mode == 3 else mode) == 0
    w = dev.World(s, mode=mode)
    w.step(300)
    st = w.stats()
    assert st["status"] == 0
    assert np.array_equal(bits(w.state()), bits(o.state()))
    assert w.hash() == o.hash()
    assert np.array_equal(w.pairs(), o.pairs()[0])


def test_world_run_to_run(dev):
    s = scenes.stress_blocks()
    hs = []
    for _ in range(2):
        w = dev.World(s)
        w.step(120)
        hs.append(w.hash())
    assert hs[0] == hs[1]


def test_world_random_pile_frames(dev, oracle_mod):
    s = scenes.random_pile(65536)
    o = oracle_mod.World(s)
    w = dev.World(s)
    for _ in range(3):
        o.step(1)
        w.step(1)
        assert np.array_equal(bits(w.state()), bits(o.state()))
    assert np.array_equal(w.pairs(), o.pairs()[0])
    ag, cg = w.contacts()
    ao, co = o.contacts()
    assert np.array_equal(ag, ao) and np.array_equal(bits(cg), bits(co))


def test_single_and_pair_scenes(dev, oracle_mod):
    """Edge sizes: one body (no tree), two bodies (root only)."""
    for n in (1, 2):
        s = scenes.determinism((1, n, 1)) if n == 1 else scenes.determinism((1, 1, 1))
        o = oracle_mod.World(s)
        w = dev.World(s)
        o.step(30)
        w.step(30)
        assert np.array_equal(bits(w.state()), bits(o.state()))


def test_pair_overflow_keeps_sorted_prefix(dev, oracle_mod):
    s = scenes.stress_blocks()
    o = oracle_mod.World(s)
    o.step(59)
    o.stage(oracle_mod.STAGE_INTEGRATE)
    st = o.state()
    o.stage(oracle_mod.STAGE_BROADPHASE)
    full, n_true = o.pairs()
    cap = n_true // 2
    bodies, shapes = dev.DeviceBodies(s), dev.DeviceShapes(s)
    bodies.set_state(st)
    bp = dev.Broadphase(s.n_bodies, cap)
    bp.build_and_query(bodies, shapes, s.bounds[0])
    assert bp.download_count() == n_true
    assert np.array_equal(bp.pairs(), full[:cap])


@pytest.mark.parametrize("n", [1, 7, 4096, 4097, 100003, 1 << 20])
def test_sort_by_key_u64(dev, n):
    import ctypes as C
    import torch
    from dyphur_b200 import capi
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 2**63, n, dtype=np.int64)
    keys[::7] = keys[0]  # duplicates: stability matters
    vals = np.arange(n, dtype=np.int32)
    kd = torch.from_numpy(keys).cuda()
    vd = torch.from_numpy(vals).cuda()
    ws_bytes = capi.lib().dyph_sort_workspace_bytes(n)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
    capi.check(capi.lib().dyph_sort_by_key_u64_u32(kd.data_ptr(), vd.data_ptr(), n, ws.data_ptr(), ws_bytes,
                                                  torch.cuda.current_stream().cuda_stream))
    order = np.argsort(keys.view(np.uint64), kind="stable")
    assert np.array_equal(kd.cpu().numpy(), keys[order])
    assert np.array_equal(vd.cpu().numpy(), vals[order])


def with_static_box(s, pos=(0.0, -0.6, 0.0)):
    """The scene plus a second static box overlapping the ground: their contact
    has w_total == 0, so it is deferred in every iteration and every solver
    iteration sweeps again."""
    import dataclasses
    n = s.n_bodies
    cat = lambda a, row: np.concatenate([a, np.asarray(row, a.dtype).reshape((1,) + a.shape[1:])])
    return dataclasses.replace(
        s, pos=cat(s.pos, pos), rot=cat(s.rot, (1, 0, 0, 0)), vel=cat(s.vel, (0, 0, 0)),
        ang=cat(s.ang, (0, 0, 0)), mass=cat(s.mass, 0.0), inertia=cat(s.inertia, np.eye(3).ravel()),
        shape=cat(s.shape, s.shape[n - 1]), flags=cat(s.flags, s.flags[n - 1]),
        targets=cat(s.targets, (0, 0, 0)), body_offset=np.array([0, n + 1], s.body_offset.dtype))


@pytest.mark.parametrize("mode", [0, 3])
def test_static_static_contact_sweeps_every_iteration(dev, oracle_mod, mode):
    s = with_static_box(scenes.stress_blocks())
    assert s.n_bodies == 1026
    o = oracle_mod.World(s)
    w = dev.World(s, mode=mode)
    for frames in (40, 80):
        assert o.step(frames, 0) == 0
        w.step(frames)
        assert np.array_equal(bits(w.state()), bits(o.state()))
    assert w.stats()["status"] == 0 and dev.device_error() == 0


@pytest.mark.parametrize("scene", ["determinism", "blocks"])
def test_colored_mode_below_threshold(dev, oracle_mod, scene):
    """Mode 2 colours at every contact count, including frames with <= 256
    contacts that the reference mode solves sequentially."""
    s = scenes.determinism((3, 3, 3)) if scene == "determinism" else scenes.stress_blocks()
    o = oracle_mod.World(s)
    w = dev.World(s, mode=2)
    assert o.step(90, oracle_mod.SOLVER_COLORED) == 0
    w.step(90)
    assert np.array_equal(bits(w.state()), bits(o.state()))


def crowd_scene():
    """A lattice of small overlapping spheres with boxes inside it: body 0 (a
    large box) has far more than 128 partners of higher index, bodies 1-8
    (mid boxes) between 33 and 128, the spheres at most 32. Every bucket path
    of the pair writer runs, and body 0's contacts force the sequential
    fallback (more than 64 colours at one body)."""
    g = np.arange(-1.9, 1.91, 0.2, dtype=np.float32)
    sph = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    mids = np.array([[x, y, z] for x in (-1.0, 1.0) for y in (-1.0, 1.0) for z in (-1.0, 1.0)], np.float32)
    pos = np.concatenate([[[0.05, 0.03, 0.02]], mids + 0.05, sph]).astype(np.float32)
    n = len(pos)
    shape = np.concatenate([[0], np.ones(8), np.full(len(sph), 2)]).astype(np.uint32)
    half = np.array([[0.6, 0.6, 0.6], [0.3, 0.3, 0.3], [0.12, 0.12, 0.12]], np.float32)
    mass = np.where(shape == 2, 4.0 / 3.0 * np.pi * 0.12 ** 3 * 500.0, 8 * half[shape].prod(1) * 500.0)
    mass = mass.astype(np.float32)
    inertia = np.zeros((n, 9), np.float32)
    for i in range(n):
        h = half[shape[i]]
        if shape[i] == 2:
            d = [0.4 * mass[i] * h[0] ** 2] * 3
        else:
            d = [mass[i] / 3.0 * (h[1] ** 2 + h[2] ** 2), mass[i] / 3.0 * (h[0] ** 2 + h[2] ** 2),
                 mass[i] / 3.0 * (h[0] ** 2 + h[1] ** 2)]
        inertia[i, [0, 4, 8]] = d
    z3 = np.zeros((n, 3), np.float32)
    rot = np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1))
    return scenes.SceneSet(
        pos=pos, rot=rot, vel=z3.copy(), ang=z3.copy(), mass=mass, inertia=inertia, shape=shape,
        flags=np.zeros(n, np.uint32), shape_type=np.array([0, 0, 1], np.uint32), shape_half=half,
        body_offset=np.array([0, n], np.uint32), shape_offset=np.array([0, 3], np.uint32),
        bounds=np.array([[-3, -3, -3, 3, 3, 3]], np.float32), targets=z3.copy(), max_pairs=1 << 18,
        max_contacts=1 << 17, dt=1.0 / 60.0, n_iters=10, friction=0.5)


def test_crowd_scene_bucket_paths(dev, oracle_mod):
    s = crowd_scene()
    o = oracle_mod.World(s)
    o.stage(oracle_mod.STAGE_INTEGRATE)
    o.stage(oracle_mod.STAGE_BROADPHASE)
    p, n_pairs = o.pairs()
    per_a = np.bincount(p[:, 0], minlength=s.n_bodies)
    assert per_a[0] > 128 and 32 < per_a[1:9].min() and per_a[1:9].max() <= 128
    assert per_a[9:].max() <= 32
    stage_parity(dev, oracle_mod, s, 0)


def test_golden_fixtures(dev):
    """Final-state hashes and counts the reference build wrote (tests/golden)."""
    from test_oracle_pins import _golden_cases, _golden_scene
    for name, g in _golden_cases().items():
        w = dev.World(_golden_scene(name), mode=g["mode"])
        w.step(g["frames"])
        assert f"{w.hash():#018x}" == g["hash"], name
        st = w.stats()
        assert st["last_pairs"] == g["pairs"] and st["last_contacts"] == g["contacts"], name
