"""Trajectory recording (dyph_world_set_trajectory): the poses every other frame,
as the reference's example loop downloads them (examples/stress_test_blocks/
main.cpp:182-197, 275-278), in .trajectory row order."""
import numpy as np
import pytest

from dyphur_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from dyphur_b200 import device
    device.require_device()
    return device


def _poses_by_frame(dev, scene, frames):
    w = dev.World(scene)
    out = []
    for _ in range(frames):
        w.step(1)
        st = w.state()
        out.append(np.ascontiguousarray(st[:7].T))
    return out


@pytest.mark.parametrize("episode", [False, True])
def test_trajectory_records_every_other_frame(dev, episode):
    import torch
    s = scenes.stress_blocks()
    frames = 21
    want = _poses_by_frame(dev, s, frames)
    w = dev.World(s)
    rec = (frames + 1) // 2
    host = torch.full((rec + 1, s.n_bodies, 7), float("nan")).pin_memory()
    w.set_trajectory(host[:rec], 2)
    if episode:
        w.capture_episode(frames)
        w.run_episode()
    else:
        w.step(7)
        w.step(frames - 7)  # the frame count carries over between calls
    torch.cuda.synchronize()
    got = host.numpy()
    for r in range(rec):
        assert np.array_equal(got[r].view(np.uint32), want[2 * r].view(np.uint32)), r
    assert np.isnan(got[rec]).all(), "nothing written past max_records"
    w.set_trajectory(None)


def test_trajectory_rejects_pageable_memory(dev):
    import torch
    from dyphur_b200 import capi
    s = scenes.determinism()
    w = dev.World(s)
    host = torch.zeros((2, s.n_bodies, 7))
    st = capi.lib().dyph_world_set_trajectory(w.h, host.data_ptr(), 2, 2)
    assert st == capi.ERR_INVALID
