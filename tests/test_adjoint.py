"""The hand-written adjoint of the fused batched frame (dyph_world_rollout_backward,
dyphur_b200.autograd.rollout) against the FP64 dual-number oracle
(oracle/dual_oracle.cpp) and central finite differences.

Scenes: the differentiable-push configuration (64 boxes of h 0.2 m resting on
a ground box, a 5 kg pusher sliding into them). Loss: sum over every scene's
64 boxes of |x_final - target|^2. Gradients: the pusher's initial velocity and
spin and every dynamic body's inverse mass, in the sequential solver order.
The dual oracle follows the float run's contact set and branches, as the
adjoint does; the tolerance is 1e-3 relative (the norm of the difference over
the norm of the oracle's gradient, per scene).
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


def _setup(dev, n_scenes=4):
    import torch
    s = scenes.push(n_scenes, seed=4)
    w = dev.World(s, mode=1)
    n = s.n_bodies
    init = w.initial
    vel = init[7:10, :n].T.clone().requires_grad_(True)
    ang = init[10:13, :n].T.clone().requires_grad_(True)
    im = w.bodies.fbuf[13, :n].clone().requires_grad_(True)
    box = np.zeros(n, bool)
    for i in range(s.n_scenes):
        box[s.body_offset[i]:s.body_offset[i] + 64] = True
    tgt = torch.from_numpy(s.targets).cuda()
    mask = torch.from_numpy(box.astype(np.float32)).cuda()
    return s, w, vel, ang, im, tgt, mask


def _loss(final, tgt, mask):
    return (((final[:3].T - tgt) ** 2).sum(1) * mask).sum()


def _dual(w, s, i, frames, at_float):
    from oracle import oracle
    b0, b1 = int(s.body_offset[i]), int(s.body_offset[i + 1])
    fb = w.bodies.fbuf.cpu().numpy()
    st = np.ascontiguousarray(w.initial[:, b0:b1].cpu().numpy())
    im = fb[13, b0:b1].copy()
    ii = np.ascontiguousarray(fb[14:20, b0:b1])
    typ = s.shape_type[s.shape[b0:b1]]
    half = np.ascontiguousarray(s.shape_half[s.shape[b0:b1]].T)
    n = b1 - b0
    pusher = 64
    params = [(k, pusher) for k in range(6)] + [(6, j) for j in range(n) if im[j] != 0]
    mask = np.zeros(n, np.uint8)
    mask[:64] = 1
    return oracle.dual_rollout(st, im, ii, typ, half, s.flags[b0:b1], frames, s.dt, s.gravity, s.n_substeps,
                               s.n_iters, s.friction, params, s.targets[b0:b1], mask, at_float=at_float), params


@pytest.mark.parametrize("frames,at_float", [(10, False), (10, True), (20, True), (30, True)])
def test_adjoint_matches_fp64_dual(dev, frames, at_float):
    """Against the FP64 dual numbers at their FP64 values (10 frames), and at the
    float values on longer horizons: once the boxes are hit the gradient grows
    fast (|g| ~ 1e2 at 30 frames, ~1e13 at 100) and FP64 and float evaluation
    points give different gradients of the same map, so the adjoint, which
    evaluates the float map, is compared with the FP64 derivative of that map."""
    import torch
    from dyphur_b200.autograd import rollout
    s, w, vel, ang, im, tgt, mask = _setup(dev)
    final = rollout(w, vel, ang, im, frames, every=5)
    _loss(final, tgt, mask).backward()
    torch.cuda.synchronize()
    g_v, g_w, g_m = vel.grad.cpu().numpy(), ang.grad.cpu().numpy(), im.grad.cpu().numpy()
    fin = final.detach().cpu().numpy()
    for i in range(s.n_scenes):
        (loss, g_dual, ff, fv), params = _dual(w, s, i, frames, at_float=at_float)
        b0, b1 = int(s.body_offset[i]), int(s.body_offset[i + 1])
        # the forward pass is the float path the oracle follows, bit for bit
        assert np.array_equal(fin[:, b0:b1].view(np.uint32), ff.view(np.uint32)), i
        p = b0 + 64
        g_gpu = [g_v[p, 0], g_v[p, 1], g_v[p, 2], g_w[p, 0], g_w[p, 1], g_w[p, 2]]
        g_gpu += [g_m[b0 + j] for k, j in params[6:]]
        g_gpu = np.array(g_gpu, np.float64)
        rel = np.linalg.norm(g_gpu - g_dual) / np.linalg.norm(g_dual)
        print(f"\nscene {i}, {frames} frames, at_float {at_float}: |g| {np.linalg.norm(g_dual):.4g}, "
              f"relative error {rel:.2e}")
        assert rel <= 1e-3, (i, rel)


def test_adjoint_matches_central_differences(dev):
    """Central differences, e = 1e-4, of the FP64 re-run (the oracle's FP64
    values along the float run's branches) for the pusher's initial velocity
    and spin and three inverse masses, against the adjoint (10 frames)."""
    import torch
    from oracle import oracle
    from dyphur_b200.autograd import rollout
    s, w, vel, ang, im, tgt, mask = _setup(dev, n_scenes=2)
    frames = 10
    final = rollout(w, vel, ang, im, frames, every=10)
    _loss(final, tgt, mask).backward()
    torch.cuda.synchronize()
    g_v, g_w, g_m = vel.grad.cpu().numpy(), ang.grad.cpu().numpy(), im.grad.cpu().numpy()
    (_, _, _, _), params = _dual(w, s, 0, frames, at_float=False)
    fb = w.bodies.fbuf.cpu().numpy()
    b1 = int(s.body_offset[1])
    st = np.ascontiguousarray(w.initial[:, :b1].cpu().numpy())
    args = (st, fb[13, :b1].copy(), np.ascontiguousarray(fb[14:20, :b1]), s.shape_type[s.shape[:b1]],
            np.ascontiguousarray(s.shape_half[s.shape[:b1]].T), s.flags[:b1], frames, s.dt, s.gravity,
            s.n_substeps, s.n_iters, s.friction, params, s.targets[:b1], (np.arange(b1) < 64).astype(np.uint8))
    eps = 1e-4
    checked = list(range(6)) + [6, 30, 60]
    for p in checked:
        lp = oracle.dual_rollout(*args, shift_param=p, shift=eps)[0]
        lm = oracle.dual_rollout(*args, shift_param=p, shift=-eps)[0]
        fd = (lp - lm) / (2 * eps)
        k, body = params[p]
        g = g_v[body, k] if k < 3 else (g_w[body, k - 3] if k < 6 else g_m[body])
        print(f"\nparameter {params[p]}: adjoint {g:.6g}, central difference {fd:.6g}")
        assert abs(g - fd) <= 1e-3 * max(abs(fd), 1e-2), (params[p], g, fd)


def test_checkpoint_spacing_does_not_change_the_gradient(dev):
    """Segments re-recorded from their checkpoints (every > 1, the last one
    shorter, or one segment longer than the rollout) give the gradient of a
    checkpoint at every frame, bit for bit."""
    import torch
    from dyphur_b200.autograd import rollout
    out = []
    for every in (1, 7, 15, 20):
        s, w, vel, ang, im, tgt, mask = _setup(dev, n_scenes=2)
        _loss(rollout(w, vel, ang, im, 15, every=every), tgt, mask).backward()
        torch.cuda.synchronize()
        out.append(np.concatenate([vel.grad.cpu().numpy().ravel(), im.grad.cpu().numpy()]))
    assert np.abs(out[0]).sum() > 0
    for o in out[1:]:
        assert np.array_equal(o.view(np.uint32), out[0].view(np.uint32))


def test_reverse_layout_does_not_change_the_gradient(dev):
    """The reverse kernel's work items and shared memory
    (dyph_world_set_adjoint_config) move only where a scene's adjoint runs and
    where its contact words live: the gradients are the same bit for bit."""
    import torch
    from dyphur_b200.autograd import rollout
    s = scenes.batch_mixed(40, 16, 512, seed=5)
    n = s.n_bodies
    dyn = torch.from_numpy((s.mass > 0).astype(np.float32)).cuda()
    out, layouts = [], set()
    for smem, teams in ((0, 1), (0, 0), (0, 2), (1, 0), (1, 1), (200 << 10, 1), (64 << 10, 2)):
        w = dev.World(s, mode=1)
        w.set_adjoint_config(smem, teams)
        cfg = w.adjoint_config()
        assert cfg["warp_scenes"] + cfg["half_scenes"] + cfg["block_scenes"] == s.n_scenes
        assert cfg["teams"] == teams and cfg["blocks_per_sm"] >= 1
        layouts.add((cfg["smem_bytes"], cfg["warp_scenes"], cfg["half_scenes"]))
        vel = w.initial[7:10, :n].T.clone().requires_grad_(True)
        ang = w.initial[10:13, :n].T.clone().requires_grad_(True)
        im = w.bodies.fbuf[13, :n].clone().requires_grad_(True)
        fin = rollout(w, vel, ang, im, 12, every=4)
        ((fin[:3].T ** 2).sum(1) * dyn).sum().backward()
        torch.cuda.synchronize()
        out.append([t.grad.cpu().numpy() for t in (vel, ang, im)])
        assert dev.device_error() == 0
    assert len(layouts) >= 5
    assert np.abs(out[0][0]).sum() > 0
    for o in out[1:]:
        for a, b in zip(o, out[0]):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_adjoint_with_deferred_contacts_matches_fp64_dual(dev):
    """Two push setups merged into one scene overlap: their static grounds
    make contacts that are deferred (w_total < 1e-10) every iteration, so every
    frame runs further sweeps in which nothing acts. The adjoint still
    differentiates the first sweep at its own pre-solve states."""
    import dataclasses

    import torch
    from dyphur_b200.autograd import rollout
    s0 = scenes.push(4, seed=4)
    o, so, b = s0.body_offset, s0.shape_offset, s0.bounds
    bounds = np.stack([np.concatenate([b[i:i + 2, :3].min(0), b[i:i + 2, 3:].max(0)]) for i in (0, 2)])
    s = dataclasses.replace(s0, body_offset=np.array([o[0], o[2], o[4]], np.uint32),
                            shape_offset=np.array([so[0], so[2], so[4]], np.uint32),
                            bounds=bounds.astype(np.float32))
    w = dev.World(s, mode=1)
    n = s.n_bodies
    vel = w.initial[7:10, :n].T.clone().requires_grad_(True)
    ang = w.initial[10:13, :n].T.clone().requires_grad_(True)
    im = w.bodies.fbuf[13, :n].clone().requires_grad_(True)
    box = np.zeros(n, bool)
    for i in range(s.n_scenes):
        box[s.body_offset[i]:s.body_offset[i] + 64] = True
    tgt = torch.from_numpy(s.targets).cuda()
    frames = 4
    final = rollout(w, vel, ang, im, frames, every=2)
    _loss(final, tgt, torch.from_numpy(box.astype(np.float32)).cuda()).backward()
    torch.cuda.synchronize()
    g_v, g_w, g_m = vel.grad.cpu().numpy(), ang.grad.cpu().numpy(), im.grad.cpu().numpy()
    from oracle import oracle
    fb = w.bodies.fbuf.cpu().numpy()
    for i in range(s.n_scenes):
        b0, b1 = int(s.body_offset[i]), int(s.body_offset[i + 1])
        sh = s.shape[b0:b1]
        mask = np.zeros(b1 - b0, np.uint8)
        mask[:64] = 1
        # the first setup's pusher and its 64 boxes' inverse masses (the oracle takes at most 96 parameters)
        params = [(k, 64) for k in range(6)] + [(6, j) for j in range(64)]
        loss, g_dual, ff, fv = oracle.dual_rollout(
            np.ascontiguousarray(w.initial[:, b0:b1].cpu().numpy()), fb[13, b0:b1].copy(),
            np.ascontiguousarray(fb[14:20, b0:b1]), s.shape_type[sh], np.ascontiguousarray(s.shape_half[sh].T),
            s.flags[b0:b1], frames, s.dt, s.gravity, s.n_substeps, s.n_iters, s.friction, params,
            s.targets[b0:b1], mask, at_float=True)
        assert np.array_equal(final.detach().cpu().numpy()[:, b0:b1].view(np.uint32), ff.view(np.uint32)), i
        p = b0 + 64
        g_gpu = [g_v[p, 0], g_v[p, 1], g_v[p, 2], g_w[p, 0], g_w[p, 1], g_w[p, 2]]
        g_gpu += [g_m[b0 + j] for k, j in params[6:]]
        g_gpu = np.array(g_gpu, np.float64)
        rel = np.linalg.norm(g_gpu - g_dual) / np.linalg.norm(g_dual)
        print(f"\nmerged scene {i}, {frames} frames: |g| {np.linalg.norm(g_dual):.4g}, relative error {rel:.2e}")
        assert rel <= 1e-3, (i, rel)
