"""CPU checks of the C ABI library: it loads without a GPU, exports every
function include/dyphur_b200.h declares, and its host-side helpers (scene
builders, BodyStore::add packing) agree with the oracle."""
import ctypes
import os
import re

import numpy as np

from dyphur_b200 import capi, scenes
from dyphur_b200._lib import LIB_PATH

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "dyphur_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dyph_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = ctypes.CDLL(LIB_PATH)
    names = header_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(capi.HEADER_SYMBOLS)


def test_status_strings_without_gpu():
    assert capi.lib().dyph_status_string(0) == b"ok"
    assert b"timed out" in capi.lib().dyph_status_string(5)


def test_device_check_reports_no_device_here():
    import torch
    if not torch.cuda.is_available():
        assert capi.lib().dyph_device_check() == capi.ERR_NO_DEVICE


def test_pack_bodies_matches_oracle(oracle_mod):
    from dyphur_b200.device import pack_bodies
    s = scenes.random_pile(2000, seed=11)
    st, im, ii, fl = pack_bodies(s)
    w = oracle_mod.World(s)
    im_o, ii_o = w.inv()
    assert np.array_equal(im.view(np.uint32), im_o.view(np.uint32))
    assert np.array_equal(ii.view(np.uint32), ii_o.view(np.uint32))
    assert np.array_equal(st.view(np.uint32), w.state().view(np.uint32))


def test_scene_builders_shapes_and_counts():
    s = scenes.stress_blocks()
    assert s.n_bodies == 1025 and s.n_scenes == 1
    assert s.max_pairs == 65536 and s.max_contacts == 16384
    assert np.allclose(s.bounds[0], [-25, -2, -25, 25, 22, 25])
    assert s.flags[-1] == 1 and s.mass[-1] == 0
    d = s.pos[:-1] - np.round(s.pos[:-1] / 0.85 - 0.5) * 0.85
    assert np.abs(s.pos[:-1, 1] - (0.5 + 0.85 * (np.arange(1024) // 64 + 1))).max() <= 0.0101
    assert d.shape == (1024, 3)
    p = scenes.random_pile(65536)
    assert p.n_bodies == 65537
    boxes = (p.shape_type[p.shape[:-1]] == 0).mean()
    assert 0.68 < boxes < 0.72
    assert np.allclose(np.linalg.norm(p.rot, axis=1), 1.0, atol=1e-6)
    b = scenes.batch(4096)
    assert b.n_scenes == 4096
    counts = np.diff(b.body_offset) - 1
    assert counts.min() >= 8 and counts.max() <= 256
    assert 40 < counts.mean() < 90


def test_scene_builders_deterministic():
    a, b = scenes.batch(64, seed=3), scenes.batch(64, seed=3)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.body_offset, b.body_offset)
    c = scenes.batch(64, seed=4)
    assert not np.array_equal(a.body_offset, c.body_offset) or not np.array_equal(a.pos, c.pos)
