"""On-disk formats of the reference's examples (dyphur_b200/formats.py), and the
stress_test_blocks drop-in (python -m dyphur_b200.run) writing them."""
import json
import os
import struct

import numpy as np
import pytest

from dyphur_b200 import formats, scenes


def test_scene_file_layout_and_round_trip(tmp_path):
    p = str(tmp_path / "s")
    idx = np.array([0, 0, 1], np.uint32)
    formats.write_scene(p, idx, [0, 1], [[0.4, 0.4, 0.4], [20.0, 0.5, 20.0]])
    raw = open(p + ".scene", "rb").read()
    assert len(raw) == 8 + 4 * 3 + 20 * 2  # scene_io.hpp:24-27
    assert struct.unpack("<II", raw[:8]) == (3, 2)
    assert struct.unpack("<IfffI", raw[20 + 20:]) == (1, 20.0, 0.5, 20.0, 0)
    i2, t2, h2 = formats.read_scene(p)
    assert np.array_equal(i2, idx) and t2.tolist() == [0, 1] and np.allclose(h2[0], 0.4)


def test_trajectory_layout_and_round_trip(tmp_path):
    p = str(tmp_path / "t")
    rng = np.random.default_rng(0)
    rec = rng.normal(size=(3, 5, 7)).astype(np.float32)
    formats.write_trajectory(p, 5, rec)  # 5 simulation frames -> 3 records (frames 0, 2, 4)
    raw = open(p + ".trajectory", "rb").read()
    assert struct.unpack("<II", raw[:8]) == (5, 5)
    assert len(raw) == 8 + rec.nbytes
    # row layout: body 1 of record 2 is x y z w qx qy qz
    off = 8 + (2 * 5 + 1) * 28
    assert np.array_equal(np.frombuffer(raw[off:off + 28], "<f4"), rec[2, 1])
    n, frames, r2 = formats.read_trajectory(p)
    assert (n, frames) == (5, 5) and np.array_equal(r2, rec)
    assert formats.trajectory_records(300) == 150 and formats.trajectory_records(5) == 3


def test_golden_and_metrics_text(tmp_path):
    p = str(tmp_path / "g")
    formats.write_golden(p, 0xcbcd209c3665c818)
    assert open(p + ".golden").read() == "cbcd209c3665c818\n"
    assert formats.read_golden(p) == 0xcbcd209c3665c818
    formats.write_metrics(p, 1025, 300, 1.0 / 60.0, 1.25, 2615.0)
    text = open(p + ".metrics.json").read()
    keys = [line.split(":")[0].strip().strip('"') for line in text.splitlines()[1:-1]]
    assert keys == ["n_bodies", "n_frames", "simulation_seconds", "wall_clock_seconds", "frames_per_second",
                    "avg_contacts_per_frame", "realtime_factor"]  # main.cpp:320-335
    m = json.loads(text)
    assert m["frames_per_second"] == 240.0 and m["simulation_seconds"] == 5.0 and m["realtime_factor"] == 4.0
    assert '"avg_contacts_per_frame": 2615.0,' in text


@pytest.mark.gpu
def test_run_writes_the_example_outputs(tmp_path, oracle_mod):
    """The drop-in run on the example's own scene (1.0 m spacing, no jitter):
    the golden equals the oracle's hash and every trajectory record the
    oracle's poses after that frame."""
    from dyphur_b200 import run
    prefix = str(tmp_path / "stb")
    frames = 24
    assert run.main([prefix, str(frames)]) == 0
    for ext in (".scene", ".trajectory", ".metrics.json", ".golden"):
        assert os.path.exists(prefix + ext), ext
    s = scenes.stress_blocks(spacing=1.0, jitter=0.0)
    o = oracle_mod.World(s)
    n, hdr_frames, rec = formats.read_trajectory(prefix)
    assert (n, hdr_frames) == (s.n_bodies, frames) and rec.shape[0] == frames // 2
    for f in range(frames):
        assert o.step(1) == 0
        if f % 2 == 0:
            want = np.ascontiguousarray(o.state()[:7].T)
            assert np.array_equal(rec[f // 2].view(np.uint32), want.view(np.uint32)), f
    assert formats.read_golden(prefix) == o.hash()
    m = formats.read_metrics(prefix)
    assert m["n_bodies"] == s.n_bodies and m["n_frames"] == frames
    idx, st, sh = formats.read_scene(prefix)
    assert np.array_equal(idx, s.shape) and np.array_equal(st, s.shape_type)
