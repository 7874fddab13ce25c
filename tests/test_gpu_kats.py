"""The reference's integrator, solver and determinism known-answer tests run
through the CUDA path (core/tests/integrator_test.cpp:26-140,
core/tests/xpbd_solver_test.cpp:74-155, core/tests/sim_determinism_test.cpp:248-256),
each also compared bit for bit with the oracle where the oracle runs the
same step."""
import numpy as np
import pytest

from dyphur_b200 import scenes
from test_oracle_pins import _single_scene

pytestmark = pytest.mark.gpu

BOX = (0, 0.5, 0.5, 0.5)
SPHERE = (1, 1.0, 1.0, 1.0)


@pytest.fixture(scope="module")
def dev():
    from dyphur_b200 import device
    device.require_device()
    return device


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _one_body(pos, vel=(0, 0, 0), ang=(0, 0, 0), mass=1.0, flags=0):
    s = _single_scene([0], [pos], [BOX], masses=[mass], flags=[flags])
    s.vel = np.asarray([vel], np.float32)
    s.ang = np.asarray([ang], np.float32)
    s.bounds = np.array([[-50, -50, -50, 50, 50, 50]], np.float32)
    return s


def _integrate_both(dev, oracle_mod, s, gravity, dt, n_sub, times=1):
    s.gravity, s.dt, s.n_substeps = tuple(gravity), dt, n_sub
    b = dev.DeviceBodies(s)
    o = oracle_mod.World(s)
    for _ in range(times):
        dev.integrate(b, gravity, dt, n_sub)
        assert o.stage(oracle_mod.STAGE_INTEGRATE) == 0
    st = b.state()
    assert np.array_equal(bits(st), bits(o.state()))
    return st


def test_static_body_does_not_move(dev, oracle_mod):
    """integrator_test.cpp:26-50."""
    st = _integrate_both(dev, oracle_mod, _one_body((1, 2, 3), mass=0.0, flags=1), (0, -9.81, 0), 1 / 60, 1)
    assert np.allclose(st[:3, 0], [1, 2, 3], atol=1e-6)


def test_free_fall_matches_symplectic_euler(dev, oracle_mod):
    """integrator_test.cpp:52-83: dt = 1 s in 60 substeps, y = 10 + g (N + 1) / 2N."""
    st = _integrate_both(dev, oracle_mod, _one_body((0, 10, 0)), (0, -9.81, 0), 1.0, 60)
    n = 60
    assert abs(st[1, 0] - (10.0 - 9.81 * (n + 1) / (2 * n))) < 1e-3
    assert abs(st[0, 0]) < 1e-5 and abs(st[2, 0]) < 1e-5


def test_constant_velocity_no_gravity(dev, oracle_mod):
    """integrator_test.cpp:85-111."""
    st = _integrate_both(dev, oracle_mod, _one_body((0, 0, 0), vel=(3, 0, 0)), (0, 0, 0), 1.0, 1)
    assert abs(st[0, 0] - 3.0) < 1e-5 and abs(st[1, 0]) < 1e-5


def test_quaternion_stays_normalised_under_spin(dev, oracle_mod):
    """integrator_test.cpp:113-140: 1 rad/s about y, 60 steps of 1/60 s in 4 substeps."""
    st = _integrate_both(dev, oracle_mod, _one_body((0, 0, 0), ang=(0, 1, 0)), (0, 0, 0), 1 / 60, 4, times=60)
    assert abs(float(np.linalg.norm(st[3:7, 0])) - 1.0) < 1e-5


def _two_spheres(vel1=(0, 0, 0), static0=False):
    s = _single_scene([0, 0], [[0, 0, 0], [0, 1.5, 0]], [SPHERE], masses=[0.0 if static0 else 1.0, 1.0],
                      flags=[1 if static0 else 0, 0])
    s.vel = np.asarray([[0, 0, 0], vel1], np.float32)
    s.bounds = np.array([[-4, -4, -4, 4, 4, 4]], np.float32)
    return s


def _narrow_and_solve(dev, s, n_iters=1):
    import torch
    bodies, shapes = dev.DeviceBodies(s), dev.DeviceShapes(s)
    np_ = dev.Narrowphase(8)
    pairs = torch.tensor([[0, 1]], dtype=torch.int32, device="cuda")
    np_.run_pairs(pairs, 1, bodies, shapes)
    assert np_.download_count()[0] == 1
    sv = dev.XpbdSolver(n_iters=n_iters, max_contacts=8, max_bodies=8)
    sv.solve(np_.contacts_view(), bodies, 1 / 60)
    return bodies.state()


def test_approaching_velocity_damped(dev):
    """xpbd_solver_test.cpp:74-109: after the solve the pair no longer approaches."""
    st = _narrow_and_solve(dev, _two_spheres(vel1=(0, -2, 0)))
    vrel_n = (st[8, 0] - st[8, 1]) * -1.0  # normal (0, -1, 0) from B toward A
    assert vrel_n >= -1e-4


def test_static_body_unmoved(dev):
    """xpbd_solver_test.cpp:112-155: only the dynamic sphere moves, upward."""
    st = _narrow_and_solve(dev, _two_spheres(static0=True))
    assert abs(st[1, 0]) < 1e-4 and st[1, 1] >= 1.0 - 1e-4


def test_large_stack_determinism_hash(dev, oracle_mod):
    """sim_determinism_test.cpp:248-256: the 256-box stack (coloured solver) over
    20 frames; the GPU hash equals the oracle's and repeats run to run."""
    s = scenes.determinism((8, 4, 8))
    hashes = []
    for _ in range(2):
        w = dev.World(s)
        w.step(20)
        hashes.append(w.hash())
    o = oracle_mod.World(s)
    assert o.step(20) == 0
    assert hashes[0] == hashes[1] == o.hash()
