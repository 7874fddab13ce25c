"""The FP64 re-run of the frame step (oracle/dual_oracle.cpp built without
tangents, dyd_fp64_run): its float trajectory is the oracle's, bit for bit,
in every solver order, so its FP64 values measure the rounding error of the
very run the GPU reproduces."""
import numpy as np
import pytest

from dyphur_b200 import scenes


def _inputs(oracle_mod, s):
    o = oracle_mod.World(s)
    im, ii = o.inv()
    st0 = o.state()
    return o, st0, im, ii, s.shape_type[s.shape], np.ascontiguousarray(s.shape_half[s.shape].T), s.flags


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_fp64_run_follows_the_float_run(oracle_mod, mode):
    s = scenes.stress_blocks()
    o, st0, im, ii, ty, h3, fl = _inputs(oracle_mod, s)
    frames = 40
    for local in (True, False):
        ep, er, fin_f, fin_v = oracle_mod.fp64_run(st0, im, ii, ty, h3, fl, frames, s.dt, s.gravity, s.n_substeps,
                                                   s.n_iters, s.friction, mode, local=local)
        if local:
            # each frame's own rounding error: present, micrometres, and the
            # final frame's is the reported one
            assert np.all(np.isfinite(fin_v)) and 0.0 < ep.max() < 1e-4 and er.max() < 1e-4
            assert abs(ep[-1] - np.sqrt(((fin_f[:3] - fin_v[:3]) ** 2).sum(0)).max()) < 1e-9
        else:
            assert ep[9] < 1e-4  # carried FP64 state: still close after 10 frames
    assert o.step(frames, mode) == 0
    assert np.array_equal(fin_f.view(np.uint32), o.state().view(np.uint32))
