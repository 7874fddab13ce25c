"""Pins of the CPU oracle (oracle/dyphur_oracle.c) before it is trusted.

1. Golden vectors from the reference's own tests (core/tests/*.cpp), checked
   against the oracle.
2. Where the reference's sources were built here (oracle/_ref), the oracle is
   compared with them stage by stage and frame by frame, bit for bit.
"""
import numpy as np
import pytest

from dyphur_b200 import scenes

GOLDEN_BOX_OMP = 0xcbcd209c3665c818  # core/tests/sim_determinism_test.cpp:224


def _world(oracle_mod, scene, which="oracle", **kw):
    return oracle_mod.World(scene, which, **kw)


def test_sim_determinism_golden(oracle_mod):
    """8 boxes + ground, 20 frames (sim_determinism_test.cpp:228-241)."""
    w1 = _world(oracle_mod, scenes.determinism())
    w2 = _world(oracle_mod, scenes.determinism())
    assert w1.step(20) == 0 and w2.step(20) == 0
    assert w1.hash() == w2.hash() == GOLDEN_BOX_OMP


def test_large_stack_run_to_run(oracle_mod):
    """256-box stack exercises the coloured path (sim_determinism_test.cpp:248-256)."""
    s = scenes.determinism((8, 4, 8))
    a, b = _world(oracle_mod, s), _world(oracle_mod, s)
    a.step(20)
    b.step(20)
    assert a.hash() == b.hash()


def test_fnv_python_matches_oracle(oracle_mod):
    w = _world(oracle_mod, scenes.determinism())
    w.step(3)
    assert oracle_mod.fnv1a64_state(w.state()) == w.hash()


def _single_scene(kind_pairs, positions, shapes, masses=None, flags=None):
    """Hand-built scene: shapes = [(type, hx, hy, hz)], kind_pairs = body->shape."""
    n = len(positions)
    s = scenes.determinism()  # template for the dataclass fields
    s.pos = np.asarray(positions, np.float32)
    s.rot = np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1))
    s.vel = np.zeros((n, 3), np.float32)
    s.ang = np.zeros((n, 3), np.float32)
    s.mass = np.asarray(masses if masses is not None else [1.0] * n, np.float32)
    s.inertia = np.tile(np.eye(3, dtype=np.float32).reshape(9), (n, 1))
    s.shape = np.asarray(kind_pairs, np.uint32)
    s.flags = np.asarray(flags if flags is not None else [0] * n, np.uint32)
    s.shape_type = np.asarray([t for t, *_ in shapes], np.uint32)
    s.shape_half = np.asarray([h for _, *h in shapes], np.float32).reshape(-1, 3)
    s.body_offset = np.array([0, n], np.uint32)
    s.shape_offset = np.array([0, len(shapes)], np.uint32)
    s.targets = np.zeros((n, 3), np.float32)
    s.max_pairs, s.max_contacts = 32, 32
    return s


def test_broadphase_three_spheres(oracle_mod):
    """broadphase_test.cpp:53-87: exactly pair (0, 1)."""
    s = _single_scene([0, 0, 0], [[0, 0, 0], [1, 0, 0], [100, 0, 0]], [(1, 1.0, 0.5, 0.5)])
    s.bounds = np.array([[-2, -2, -2, 102, 2, 2]], np.float32)
    w = _world(oracle_mod, s)
    w.stage(oracle_mod.STAGE_BROADPHASE)
    pairs, n = w.pairs()
    assert n == 1 and pairs.tolist() == [[0, 1]]


def test_broadphase_four_spheres_all_pairs(oracle_mod):
    """broadphase_test.cpp:90-131: all 6 unique a < b pairs."""
    s = _single_scene([0] * 4, [[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0], [0, 0, 0.5]], [(1, 1.0, 0.5, 0.5)])
    s.bounds = np.array([[-2, -2, -2, 2, 2, 2]], np.float32)
    w = _world(oracle_mod, s)
    w.stage(oracle_mod.STAGE_BROADPHASE)
    pairs, n = w.pairs()
    assert n == 6
    assert sorted(map(tuple, pairs.tolist())) == [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def test_broadphase_disjoint(oracle_mod):
    s = _single_scene([0, 0], [[0, 0, 0], [5, 0, 0]], [(1, 0.4, 0.5, 0.5)])
    s.bounds = np.array([[-1, -1, -1, 6, 1, 1]], np.float32)
    w = _world(oracle_mod, s)
    w.stage(oracle_mod.STAGE_BROADPHASE)
    assert w.pairs()[1] == 0


NP_CASES = [
    # narrowphase_test.cpp:217-247 sphere-sphere: depth .5, n (-1,0,0), p (.75,0,0)
    ("sphere_sphere", [0, 0], [[0, 0, 0], [1.5, 0, 0]], [(1, 1.0, 0.5, 0.5)],
     (0.5, (-1, 0, 0), (0.75, 0, 0))),
    # :276-310 sphere-box: depth .2, n (-1,0,0), p (1,0,0)
    ("sphere_box", [0, 1], [[0, 0, 0], [1.3, 0, 0]], [(0, 1.0, 1.0, 1.0), (1, 0.5, 0.5, 0.5)],
     (0.2, (-1, 0, 0), (1.0, 0, 0))),
    # :314-343 box-box face: depth .2, n (-1,0,0), p.x 1
    ("box_box", [0, 0], [[0, 0, 0], [1.8, 0, 0]], [(0, 1.0, 1.0, 1.0)], (0.2, (-1, 0, 0), (1.0, None, None))),
]


@pytest.mark.parametrize("name,shape_of,pos,shapes,expect", NP_CASES, ids=[c[0] for c in NP_CASES])
def test_narrowphase_kats(oracle_mod, name, shape_of, pos, shapes, expect):
    s = _single_scene(shape_of, pos, shapes)
    s.bounds = np.array([[-5, -5, -5, 5, 5, 5]], np.float32)
    w = _world(oracle_mod, s)
    w.stage(oracle_mod.STAGE_BROADPHASE)
    w.stage(oracle_mod.STAGE_NARROWPHASE)
    ab, p7 = w.contacts()
    assert len(ab) == 1
    depth, nrm, pt = expect
    assert abs(p7[0, 6] - depth) < 1e-4
    assert np.allclose(p7[0, 3:6], nrm, atol=1e-4)
    for k, v in enumerate(pt):
        if v is not None:
            assert abs(p7[0, k] - v) < 1e-4


@pytest.mark.parametrize("shapes,pos", [([(1, 1.0, 0.5, 0.5)], [[0, 0, 0], [3, 0, 0]]),
                                        ([(0, 1.0, 1.0, 1.0)], [[0, 0, 0], [5, 0, 0]])])
def test_narrowphase_no_contact(oracle_mod, shapes, pos):
    s = _single_scene([0, 0], pos, shapes)
    s.bounds = np.array([[-6, -6, -6, 6, 6, 6]], np.float32)
    w = _world(oracle_mod, s)
    w.stage(oracle_mod.STAGE_BROADPHASE)
    w.stage(oracle_mod.STAGE_NARROWPHASE)
    assert len(w.contacts()[0]) == 0


def test_integrator_free_fall(oracle_mod):
    """integrator_test.cpp:52-83: 60 substeps of 1/60 s from rest."""
    s = _single_scene([0], [[0, 10, 0]], [(1, 0.1, 0.1, 0.1)])
    s.bounds = np.array([[-20, -20, -20, 20, 20, 20]], np.float32)
    s.dt, s.n_substeps = 1.0, 60
    w = _world(oracle_mod, s)
    w.stage(oracle_mod.STAGE_INTEGRATE)
    st = w.state()
    expected = 10.0 + (-9.81) * 61 / 120
    assert abs(st[1, 0] - expected) < 1e-3 and abs(st[0, 0]) < 1e-5


def test_solver_sphere_pair_separates(oracle_mod):
    """xpbd_solver_test.cpp:182-215."""
    s = _single_scene([0, 0], [[0, 0, 0], [0, 1.5, 0]], [(1, 1.0, 0.5, 0.5)])
    s.bounds = np.array([[-5, -5, -5, 5, 5, 5]], np.float32)
    s.n_iters = 1
    w = _world(oracle_mod, s)
    for st in (oracle_mod.STAGE_BROADPHASE, oracle_mod.STAGE_NARROWPHASE, oracle_mod.STAGE_SOLVE):
        w.stage(st)
    y = w.state()[1]
    assert y[1] - y[0] >= 2.0 - 1e-3


def test_solver_colored_equals_serial_on_independent_pairs(oracle_mod):
    """xpbd_solver_test.cpp:302-375: 300 disjoint sphere pairs, coloured == serial bit for bit."""
    n_pairs = 300
    pos = []
    for k in range(n_pairs):
        pos += [[0, 10.0 * k, 0], [0, 10.0 * k + 0.8, 0]]
    s = _single_scene([0] * (2 * n_pairs), pos, [(1, 0.5, 0.5, 0.5)])
    s.bounds = np.array([[-10, -10, -10, 10, 3010, 10]], np.float32)
    s.max_pairs, s.max_contacts = 4096, 4096
    out = {}
    for mode in (oracle_mod.SOLVER_REFERENCE, oracle_mod.SOLVER_SERIAL):
        w = _world(oracle_mod, s)
        for st in (oracle_mod.STAGE_BROADPHASE, oracle_mod.STAGE_NARROWPHASE):
            w.stage(st)
        assert len(w.contacts()[0]) == n_pairs
        w.stage(oracle_mod.STAGE_SOLVE, mode)
        out[mode] = w.state()
    assert np.array_equal(out[0].view(np.uint32), out[1].view(np.uint32))


def test_oracle_f16_matches_numpy(oracle_mod):
    import ctypes
    lib = ctypes.CDLL(oracle_mod.build_oracle())
    lib.dyo_f32_to_f16.restype = ctypes.c_uint16
    lib.dyo_f32_to_f16.argtypes = [ctypes.c_float]
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.normal(0, 30, 4000), rng.normal(0, 1e-5, 1000), [0.0, -0.0, 65504.0, 65520.0,
                                                                                  1e-8, -2.5e-7, 6.1e-5]])
    vals = vals.astype(np.float32)
    got = np.array([lib.dyo_f32_to_f16(float(v)) for v in vals], np.uint16)
    assert np.array_equal(got, vals.astype(np.float16).view(np.uint16))


ref_only = pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).ref_available()",
                              reason="reference sources not built here (oracle/_ref)")


@ref_only
@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_matches_reference_build_blocks(oracle_mod, mode):
    """Stress-block scene (1024 boxes, 0.85 m, jitter): every 25 frames, state,
    pair list and contact list bit for bit, for 150 frames."""
    s = scenes.stress_blocks()
    o, r = _world(oracle_mod, s), _world(oracle_mod, s, "ref")
    for f in range(150):
        assert o.step(1, mode) == 0 and r.step(1, mode) == 0
        if f % 25 == 24:
            assert np.array_equal(o.state().view(np.uint32), r.state().view(np.uint32)), f
            po, npo = o.pairs()
            pr, npr = r.pairs()
            assert npo == npr and np.array_equal(po, pr)
            (ao, co), (ar, cr) = o.contacts(), r.contacts()
            assert np.array_equal(ao, ar) and np.array_equal(co.view(np.uint32), cr.view(np.uint32))
            bo, br = o.bvh(), r.bvh()
            for k in bo:
                assert np.array_equal(bo[k], br[k]), k
            if mode == 0 and len(ao) > 256:
                assert np.array_equal(o.colors(), r.colors())


@ref_only
def test_oracle_matches_reference_build_pile(oracle_mod):
    """Random 4096-body pile (boxes + spheres, random rotations), 6 frames."""
    s = scenes.random_pile(4096, seed=7)
    o, r = _world(oracle_mod, s), _world(oracle_mod, s, "ref")
    for _ in range(6):
        o.step(1)
        r.step(1)
        assert np.array_equal(o.state().view(np.uint32), r.state().view(np.uint32))
        assert np.array_equal(o.pairs()[0], r.pairs()[0])


def _golden_cases():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")) as f:
        return json.load(f)["cases"]


def _golden_scene(name):
    from dyphur_b200 import scenes
    if name.startswith("determinism"):
        return scenes.determinism()
    if name.startswith("blocks"):
        return scenes.stress_blocks()
    return scenes.random_pile(4096, seed=7)


def test_restatement_matches_reference_golden_fixtures(oracle_mod):
    """The C restatement against the fixtures the reference build wrote."""
    for name, g in _golden_cases().items():
        w = oracle_mod.World(_golden_scene(name))
        assert w.step(g["frames"], g["mode"]) == 0
        assert f"{w.hash():#018x}" == g["hash"], name
        assert w.pairs()[1] == g["pairs"] and len(w.contacts()[0]) == g["contacts"], name
