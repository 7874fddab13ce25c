"""Knobs of the fused batched frame and their autotuner (dyph_world_autotune):
every configuration gives the same frames bit for bit, the tuner leaves the
world's state and statistics as it found them, and its choice is cached per
batch profile."""
import numpy as np
import pytest

from dyphur_b200 import capi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from dyphur_b200 import device
    device.require_device()
    return device


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("mode", [capi.SOLVER_SEQUENTIAL, capi.SOLVER_COLORED])
def test_every_config_gives_the_same_frames(dev, mode):
    s = scenes.batch(192, 8, 256, seed=11)
    ref = dev.World(s, mode=mode)
    ref.step(30)
    want = ref.state()
    need = ref.fused_config()["smem_bytes"]
    seen = set()
    for cap, teams, regs in ((0, 2, 4), (0, 1, 4), (0, 0, 5), (48 << 10, 2, 5), (48 << 10, 1, 6), (32 << 10, 2, 6),
                             (1, 0, 6)):
        w = dev.World(s, mode=mode)
        w.set_fused_config(cap, teams, regs)
        cfg = w.fused_config()
        assert cfg["smem_bytes"] <= need and cfg["teams"] == teams and cfg["register_blocks"] == regs
        assert cfg["warp_scenes"] + cfg["half_scenes"] + cfg["block_scenes"] == s.n_scenes
        assert (teams >= 2) or cfg["half_scenes"] == 0
        seen.add((cfg["smem_bytes"], cfg["warp_scenes"], cfg["half_scenes"]))
        w.step(30)
        assert np.array_equal(bits(w.state()), bits(want)), (cap, teams)
        assert w.stats()["status"] == 0 and dev.device_error() == 0
    assert len(seen) >= 5 and any(k[2] > 0 for k in seen)  # the configurations really differ


def test_autotune_keeps_state_and_caches(dev):
    s = scenes.batch(256, 8, 256, seed=12)
    w = dev.World(s, mode=capi.SOLVER_SEQUENTIAL)
    w.step(5)
    before = w.state()
    stats = w.stats()
    cfg = w.autotune(8)
    assert cfg["candidates"] >= 2 and cfg["ms_per_frame"] > 0 and cfg["blocks_per_sm"] >= 1
    assert np.array_equal(bits(w.state()), bits(before)) and w.stats() == stats
    w.step(25)
    plain = dev.World(s, mode=capi.SOLVER_SEQUENTIAL)
    plain.step(30)
    assert np.array_equal(bits(w.state()), bits(plain.state()))
    again = dev.World(s, mode=capi.SOLVER_SEQUENTIAL).autotune(8)
    assert again["candidates"] == 0 and again["smem_bytes"] == cfg["smem_bytes"]
    assert dev.device_error() == 0


def test_worlds_with_different_shared_memory_step_side_by_side(dev):
    """The fused kernels' shared-memory limit is the kernel's, not the world's:
    a world set up with less shared memory after another does not make the
    other's launches fail."""
    s = scenes.batch(160, 8, 256, seed=13)
    big = dev.World(s, mode=capi.SOLVER_SEQUENTIAL)
    big.step(3)
    small = dev.World(s, mode=capi.SOLVER_SEQUENTIAL)
    small.set_fused_config(1, 0, 4)  # the floor: bodies plus 64 contacts' words
    assert small.fused_config()["smem_bytes"] < big.fused_config()["smem_bytes"]
    small.step(3)
    big.step(12)
    small.step(12)
    assert np.array_equal(bits(big.state()), bits(small.state()))
    assert dev.device_error() == 0
