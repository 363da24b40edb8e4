"""Adjoint of a moving run: the motion checkpoints (pppm_checkpoint_*), the cache-state blobs
(pppm_save_cache_state / pppm_restore_cache_state) and pppm_b200.autograd.moving_listener_signal.

A moving run is still linear in the accelerations for a prescribed motion, series = A acc, with
every step using the tables of its motion frame.  Those tables depend on the whole motion (the
grid cache recomputes only the triangles that moved past its threshold, the face cache keeps the
records of pairs it has seen), so the backward rebuilds them frame by frame from checkpoints.  Checked:

  * a rewind to a motion checkpoint (or a blob restore, host or device memory) followed by the
    frame's update_mesh reproduces that frame's tables byte for byte (FP32: fp16 records with
    their scales; FP64), on a breathing sphere whose face records are rewritten every frame, and
    a replayed run reproduces the original run's listener series bit for bit;
  * stepping or a new checkpoint after a rewind without update_mesh is refused, as is a rewind
    to a dropped checkpoint or a blob of another mesh;
  * FP64: <g, A x> = <A^T g, x> to 1e-10 and the Jacobian column by column (unit impulses) to 1e-10,
    across motion frames that move triangles into other cells;
  * the gradient does not depend on the checkpoint spacing (bit-identical);
  * each precision's gradient against central differences of its own forward (dyadic inputs and
    directions, so the difference quotient is centred exactly: FP64 1e-9, FP32 1e-3), the FP32
    gradient against the FP64 one.

When PPPM_METRICS_DIR is set the measured errors go to adjoint_moving_metrics.json there.
"""
import json
import os

import numpy as np
import pytest

from helpers import dyadic, sphere_small
from pppm_b200 import PPPMError, Solver, scenes

pytestmark = pytest.mark.gpu

METRICS = {}
TABLES = ("grid_cache", "face_pairs", "face_cache", "n3_cells", "n3_tris", "b4_cells", "b4_tris", "n4_tris",
          "interp", "tri_cells")


def _record(key, value):
    METRICS[key] = value
    d = os.environ.get("PPPM_METRICS_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "adjoint_moving_metrics.json"), "w") as f:
            json.dump(METRICS, f, indent=1)


def _frames(v0, h, nframes, every):
    """a rotation of 0.15 rad and a drift of (0.35, 0.2, -0.1) cells per frame: triangles change
    cells and meet new neighbours within a few frames"""
    out = []
    for k in range(nframes):
        R = scenes.rotation_matrix([0.3, 0.5, 0.8], 0.15 * k)
        v = v0.astype(np.float64) @ R.T + np.array([0.35, 0.2, -0.1]) * float(h) * k
        out.append((k * every, v.astype(np.float32)))
    return out


def _breathing_frames(v0, h, nframes, every):
    """the drift of _frames with the sphere scaled by 1 + 0.03 k about its centre: every face
    pair's distance changes by more than 1 % per frame, so the face cache rewrites its records
    in place (the case the motion checkpoints log)"""
    c = v0.astype(np.float64).mean(0)
    out = []
    for k in range(nframes):
        v = (v0.astype(np.float64) - c) * (1 + 0.03 * k) + c + np.array([0.35, 0.2, -0.1]) * float(h) * k
        out.append((k * every, v.astype(np.float32)))
    return out


def _solver(precision, res=20, sub=1):
    v, f, h, mn, dt = sphere_small(res, sub)
    s = Solver(res, h, dt, mn, precision=precision)
    s.set_mesh(v, f)
    s.add_listener(res - 4, res - 4, res - 4)
    c = s.dump("n3_cells").reshape(-1, 4)[0]
    s.add_listener(int(c[0]), int(c[1]), int(c[2]))
    s.add_listener(1, res // 2, res // 3)
    return s, v, h


def _tables(s):
    return {k: s.dump(k).tobytes() for k in TABLES}


def _run_frames(s, x, frames):
    bounds = [f[0] for f in frames] + [len(x)]
    for k, (_, v) in enumerate(frames):
        if k:
            s.update_mesh(v)
        s.step(x[bounds[k]: bounds[k + 1]])


def _to_start(s, ckpt0, frames):
    """frame 0's tables (rebuilt from its checkpoint), zero fields, no recorded samples"""
    s.restore_cache_state(ckpt0)
    s.update_mesh(frames[0][1])
    s.reset_fields()
    s.rewind_listeners()


def _replay(s, ckpt0, x, frames):
    """the series of a run over x from the zero state"""
    _to_start(s, ckpt0, frames)
    _run_frames(s, x, frames)
    return s.series(0, len(x)).astype(np.float64)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_checkpoint_rewind_restores_the_frame_tables(gpu, precision):
    """motion checkpoints (pppm_checkpoint_*): the pool stays in place and its rewrites are
    logged; a rewind plus the frame's update_mesh gives the frame's tables byte for byte"""
    s, v0, h = _solver(precision)
    frames = _breathing_frames(v0, h, 6, 10)
    x = np.random.default_rng(11).standard_normal((60, s.nt)).astype(np.float32)
    bounds = [f[0] for f in frames] + [60]
    want, ids = {}, {}
    for k, (_, v) in enumerate(frames):
        if k:
            s.update_mesh(v)
        want[k] = _tables(s)
        if k in (0, 2, 4):
            ids[k] = s.checkpoint_push()
        s.step(x[bounds[k]: bounds[k + 1]])
    series = s.series(0, 60).astype(np.float64)
    count, held = s.checkpoint_info()
    assert count == 3 and held > 0
    assert want[1]["face_cache"] != want[2]["face_cache"]  # records rewritten in place
    for ck, frames_to_check in ((4, (5, 4)), (2, (3, 2))):
        for k in frames_to_check:
            s.checkpoint_rewind(ids[ck])
            with pytest.raises(PPPMError):
                s.step(x[:1])  # the lists still describe the geometry before the rewind
            with pytest.raises(PPPMError):
                s.checkpoint_push()
            for j in range(ck, k + 1):
                s.update_mesh(frames[j][1])
            got = _tables(s)
            assert [t for t in TABLES if got[t] != want[k][t]] == [], (ck, k)
    assert s.checkpoint_info()[0] == 2  # rewinding to checkpoint 2 dropped the one of frame 4
    # from frame 0 again: every frame's tables and the whole series as in the first run
    s.checkpoint_rewind(ids[0])
    s.update_mesh(frames[0][1])
    s.reset_fields()
    s.rewind_listeners()
    for k, (_, v) in enumerate(frames):
        if k:
            s.update_mesh(v)
        got = _tables(s)
        assert [t for t in TABLES if got[t] != want[k][t]] == [], k
        s.step(x[bounds[k]: bounds[k + 1]])
    assert np.array_equal(s.series(0, 60).astype(np.float64), series)
    with pytest.raises(PPPMError):
        s.checkpoint_rewind(3)
    s.checkpoint_clear()
    assert s.checkpoint_info()[0] == 0 and s.checkpoint_info()[1] > 0  # the arena is kept
    s.checkpoint_clear(release=True)
    assert s.checkpoint_info() == (0, 0)
    s.close()


@pytest.mark.parametrize("precision,on_device", [("fp32", True), ("fp64", False), ("fp32", False)])
def test_cache_state_restores_the_frame_tables(gpu, precision, on_device):
    s, v0, h = _solver(precision)
    frames = _breathing_frames(v0, h, 6, 10)
    x = np.random.default_rng(1).standard_normal((60, s.nt)).astype(np.float32)
    ckpt0 = s.save_cache_state()
    bounds = [f[0] for f in frames] + [60]
    want, ckpt = {}, {}
    for k, (_, v) in enumerate(frames):
        if k:
            s.update_mesh(v)
        want[k] = _tables(s)
        ckpt[k] = s.save_cache_state(on_device=on_device)
        s.step(x[bounds[k]: bounds[k + 1]])
    series = s.series(0, 60).astype(np.float64)
    # the motion reaches new cells and new face pairs
    assert want[0]["tri_cells"] != want[5]["tri_cells"]
    assert want[0]["face_pairs"] != want[5]["face_pairs"]
    # each frame's tables from the checkpoint of frame 2 plus the update_mesh calls up to it
    for k in (2, 3, 5):
        s.restore_cache_state(ckpt[2])
        with pytest.raises(PPPMError):
            s.step(x[:1])  # the lists still describe the geometry before the restore
        for j in range(2, k + 1):
            s.update_mesh(frames[j][1])
        got = _tables(s)
        assert [t for t in TABLES if got[t] != want[k][t]] == []
    # a replayed run is the run
    assert np.array_equal(_replay(s, ckpt0, x, frames), series)
    # a blob of another mesh
    o, _, _ = _solver(precision, sub=0)
    with pytest.raises(PPPMError):
        o.restore_cache_state(ckpt[2])
    o.close()
    s.close()


def test_moving_dot_product_and_spacing_fp64(gpu):
    import torch

    from pppm_b200.autograd import moving_listener_signal

    s, v0, h = _solver("fp64")
    frames = _frames(v0, h, 5, 15)
    n = 75
    rng = np.random.default_rng(2)
    x32 = rng.standard_normal((n, s.nt)).astype(np.float32)
    ckpt0 = s.save_cache_state()
    x = torch.tensor(x32.astype(np.float64), device="cuda", requires_grad=True)
    g = torch.tensor(rng.standard_normal((n, s.n_listeners)), device="cuda")
    grads = []
    for spacing in (30, 1, 10 ** 9):
        _to_start(s, ckpt0, frames)
        sig = moving_listener_signal(s, x, frames, checkpoint_steps=spacing)
        (gx,) = torch.autograd.grad(sig, x, g)
        grads.append(gx.cpu().numpy())
        y = sig.detach().cpu().numpy()
    gn = g.cpu().numpy()
    lhs, rhs = float(np.sum(gn * y)), float(np.sum(grads[0] * x32.astype(np.float64)))
    scale = float(np.sum(np.abs(gn * y)))
    _record("moving_dot_product_fp64_rel", abs(lhs - rhs) / scale)
    assert abs(lhs - rhs) <= 1e-10 * scale, (lhs, rhs)
    assert np.array_equal(grads[0], grads[1]) and np.array_equal(grads[0], grads[2])
    # the run the autograd forward took is the run from the zero state
    assert np.array_equal(y, _replay(s, ckpt0, x32, frames))
    s.close()


def test_moving_jacobian_fp64(gpu):
    import torch

    from pppm_b200.autograd import moving_listener_signal

    s, v0, h = _solver("fp64", res=16, sub=0)
    frames = _frames(v0, h, 4, 4)
    n, nt, nl = 16, s.nt, s.n_listeners
    ckpt0 = s.save_cache_state()
    J = np.zeros((n, nl, n, nt))
    e = np.zeros((n, nt), np.float32)
    for k in range(n):
        for j in range(nt):
            e[k, j] = 1.0
            J[:, :, k, j] = _replay(s, ckpt0, e, frames)
            e[k, j] = 0.0
    rng = np.random.default_rng(3)
    worst = 0.0
    for trial in range(3):
        g = rng.standard_normal((n, nl))
        want = np.einsum("sl,slkj->kj", g, J)
        _to_start(s, ckpt0, frames)
        x = torch.zeros((n, nt), dtype=torch.float64, device="cuda", requires_grad=True)
        sig = moving_listener_signal(s, x, frames, checkpoint_steps=8)
        (got,) = torch.autograd.grad(sig, x, torch.tensor(g, device="cuda"))
        err = np.abs(got.cpu().numpy() - want).max() / np.abs(want).max()
        worst = max(worst, float(err))
    _record("moving_jacobian_fp64_max_rel", worst)
    assert worst <= 1e-10
    s.close()


def test_moving_gradient_vs_finite_differences(gpu):
    import torch

    from pppm_b200.autograd import moving_listener_signal

    n = 90
    rng = np.random.default_rng(4)
    res = {}
    for precision in ("fp64", "fp32"):
        s, v0, h = _solver(precision, res=24, sub=2)
        frames = _frames(v0, h, 6, 15)
        ckpt0 = s.save_cache_state()
        if precision == "fp64":
            acc = dyadic(rng, (n, s.nt))
            # a target on the signal's scale: the difference quotient then does not cancel
            base = _replay(s, ckpt0, acc, frames)
            target = rng.standard_normal((n, s.n_listeners)) * base.std()
            dirs = [dyadic(rng, acc.shape) for _ in range(8)]
            _to_start(s, ckpt0, frames)
        # float64 leaves for the FP64 scheme: the gradient comes back in the leaf's dtype
        x = torch.tensor(acc.astype(s.real), device="cuda", requires_grad=True)
        sig = moving_listener_signal(s, x, frames, checkpoint_steps=40)
        loss = ((sig.double() - torch.tensor(target, device="cuda")) ** 2).sum()
        loss.backward()
        grad = x.grad.cpu().numpy().astype(np.float64)

        def f(z):
            return float(np.sum((_replay(s, ckpt0, z, frames) - target) ** 2))

        worst = 0.0
        for v in dirs:
            eps = 0.125
            xp, xm = acc + np.float32(eps) * v, acc - np.float32(eps) * v  # exact: dyadic inputs
            fd = (f(xp) - f(xm)) / (2 * eps)
            an = float(np.sum(grad * v.astype(np.float64)))
            worst = max(worst, abs(fd - an) / max(abs(fd), 1e-300))
        res[precision] = (grad, worst)
        s.close()
    rel = float(np.linalg.norm(res["fp32"][0] - res["fp64"][0]) / np.linalg.norm(res["fp64"][0]))
    _record("moving_fp64_vs_fd_max_rel", res["fp64"][1])
    _record("moving_fp32_vs_fd_max_rel", res["fp32"][1])
    _record("moving_fp32_vs_fp64_rel_l2", rel)
    assert res["fp64"][1] <= 1e-9
    assert res["fp32"][1] <= 1e-3
    assert rel <= 1e-2
