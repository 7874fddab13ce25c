"""Batched scenes in one world (dyph_world_set_scenes).

Every scene of a batch must evolve bit for bit as it does stepped alone in the
same solver mode: its bodies never pair with another scene's, its contacts are
a contiguous run of the contact list, and one thread block runs the
reference's solve on that run with the scene's own contact indices.
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


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_batched_scenes_match_oracle_per_scene(dev, oracle_mod, mode):
    """Every scene of a batch, solved one scene per block, evolves bit for bit
    as the oracle steps it alone in the same mode: 0 the reference's order
    (sequential at <= 256 contacts, else JP colours of the scene's own contact
    indices), 1 sequential, 2 JP colours at every count."""
    s = scenes.batch(40, 8, 200, seed=11)
    w = dev.World(s, mode=mode)
    w.step(80)
    assert w.stats()["status"] == 0 and dev.device_error() == 0
    hb = w.scene_hashes()
    for i in range(s.n_scenes):
        o = oracle_mod.World(s.scene(i))
        assert o.step(80, mode) == 0
        assert o.hash() == int(hb[i]), (mode, i)
    if mode == 2:
        assert w.solver_stats()["path"] == 2 and w.solver_stats()["colors"] > 0


def test_batched_mixed_scenes_large_and_empty(dev, oracle_mod):
    """Mixed boxes / spheres with random rotations, up to 512 bodies a scene:
    the largest scenes' contact words spill from shared memory to the global
    scratch, and scenes without contacts in a frame (bodies still falling)
    must not be renormalised, as a scene stepped alone is not."""
    s = scenes.batch_mixed(10, 16, 512, seed=7)
    assert (np.diff(s.body_offset) > 400).any()
    for mode in (0, 1):
        w = dev.World(s, mode=mode)
        hb = []
        for frames in (3, 40):
            w.step(frames)
            hb.append(w.scene_hashes())
        assert w.stats()["status"] == 0 and dev.device_error() == 0
        for i in range(s.n_scenes):
            o = oracle_mod.World(s.scene(i))
            for k, frames in enumerate((3, 40)):
                assert o.step(frames, mode) == 0
                assert o.hash() == int(hb[k][i]), (mode, i, k)


def concat_scenes(parts):
    """Independent scenes side by side as one scene set (a batch)."""
    import dataclasses
    body_off, shape_off = [0], [0]
    for p in parts:
        body_off.append(body_off[-1] + p.n_bodies)
        shape_off.append(shape_off[-1] + len(p.shape_type))
    cat = lambda f: np.concatenate([getattr(p, f) for p in parts])
    shape = np.concatenate([p.shape + np.uint32(shape_off[i]) for i, p in enumerate(parts)]).astype(np.uint32)
    return dataclasses.replace(
        parts[0], pos=cat("pos"), rot=cat("rot"), vel=cat("vel"), ang=cat("ang"), mass=cat("mass"),
        inertia=cat("inertia"), shape=shape, flags=cat("flags"), shape_type=cat("shape_type"),
        shape_half=cat("shape_half"), body_offset=np.array(body_off, np.uint32),
        shape_offset=np.array(shape_off, np.uint32), bounds=cat("bounds"), targets=cat("targets"),
        max_pairs=sum(p.max_pairs for p in parts), max_contacts=sum(p.max_contacts for p in parts))


def test_batched_dense_scene_spills_contact_words(dev, oracle_mod):
    """A lattice of 1000 overlapping spheres (about 3000 contacts, more than a
    block's shared memory holds next to its bodies) between two small scenes:
    that scene's per-contact words live in the global scratch."""
    from test_gpu_parity import crowd_scene
    dense = crowd_scene()
    keep = np.abs(dense.pos).max(1) < 1.0  # the inner 10 x 10 x 10 spheres and the boxes inside them
    keep &= dense.shape == 2
    idx = np.nonzero(keep)[0]
    import dataclasses
    dense = dataclasses.replace(dense, pos=dense.pos[idx], rot=dense.rot[idx], vel=dense.vel[idx], ang=dense.ang[idx],
                                mass=dense.mass[idx], inertia=dense.inertia[idx], shape=dense.shape[idx],
                                flags=dense.flags[idx], targets=dense.targets[idx],
                                body_offset=np.array([0, len(idx)], np.uint32), max_pairs=1 << 16,
                                max_contacts=1 << 14)
    assert dense.n_bodies == 1000
    s = concat_scenes([scenes.determinism((3, 3, 3)), dense, scenes.determinism((2, 2, 2))])
    for mode in (0, 1):
        w = dev.World(s, mode=mode)
        w.step(2)
        assert w.contacts()[0].shape[0] > 2500
        w.step(8)
        assert w.stats()["status"] == 0 and dev.device_error() == 0
        hb = w.scene_hashes()
        for i in range(s.n_scenes):
            o = oracle_mod.World(s.scene(i))
            assert o.step(10, mode) == 0
            assert o.hash() == int(hb[i]), (mode, i)


def test_batched_lists_match_oracle_per_scene(dev, oracle_mod):
    """The fused frame's compacted lists (dyph_world_sync_lists): pairs,
    contact rows and JP colours of every scene equal the oracle's for the
    scene stepped alone, in scene order."""
    s = scenes.batch(24, 8, 200, seed=13)
    w = dev.World(s, mode=0)
    w.step(60)
    pairs = w.pairs()
    ab, p7 = w.contacts()
    cols, _ = w.colors(len(ab))
    po = pc = 0
    n_colored = 0
    for i in range(s.n_scenes):
        o = oracle_mod.World(s.scene(i))
        assert o.step(60, 0) == 0
        off = np.uint32(s.body_offset[i])
        op, _ = o.pairs()
        assert np.array_equal(pairs[po:po + len(op)], op + off), i
        po += len(op)
        oab, op7 = o.contacts()
        assert np.array_equal(ab[pc:pc + len(oab)], oab + off), i
        assert np.array_equal(p7[pc:pc + len(oab)].view(np.uint32), op7.view(np.uint32)), i
        oc = o.colors()
        assert np.array_equal(cols[pc:pc + len(oab)], oc), i
        n_colored += int(not np.all(oc == 0xFFFFFFFF))
        pc += len(oab)
    assert po == len(pairs) and pc == len(ab)
    assert n_colored > 0, "no scene took the coloured order"
