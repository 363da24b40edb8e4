"""Batched scenes (pppm_batch_*) against the same scenes stepped one by one.

The batch runs every scene's stage code on that scene's own arrays, in the same order, so the
listener series and the grids must be bit-identical to stepping each scene alone, through
uneven step counts (scenes dropping out of the batch), graph remainders and later single-scene
steps.
"""
import numpy as np
import pytest

from helpers import edge_sphere, sine_acc
from pppm_b200 import Batch, PPPMError, Solver, scenes

pytestmark = pytest.mark.gpu


def _scene(res, sub, seed, pml_width=0):
    rng = np.random.default_rng(seed)
    v, f = scenes.icosphere(sub)
    v = v * (1 + 0.08 * rng.uniform(-1, 1, (len(v), 1)))
    v = (v * 0.1).astype(np.float32)
    h, mn = scenes.grid_for_bbox(v.min(0), v.max(0), res, 2.0)
    mn = (mn + np.array([0.137, 0.291, 0.0713]) * h).astype(np.float32)
    dt = np.float32(0.5 * h / (np.sqrt(3) * 340.3))
    s = Solver(res, h, dt, mn, pml_width=pml_width)
    s.set_mesh(v, f)
    s.add_listener(res - 4, res - 4, res - 4)
    s.add_listener(res // 3, res // 2, res - 5)
    return s, f, dt


CASES = [(20, 1, 1, 37), (24, 2, 2, 50), (28, 1, 3, 13), (24, 2, 4, 50), (32, 2, 5, 21)]


def _make():
    out = []
    for res, sub, seed, steps in CASES:
        s, f, dt = _scene(res, sub, seed)
        acc = sine_acc(steps + 30, len(f), 900.0 + 100 * seed, dt)
        out.append((s, acc, steps))
    return out


def test_batch_matches_single_scenes(gpu):
    alone = _make()
    for s, acc, steps in alone:
        s.step(acc[:steps])
    together = _make()
    b = Batch([s for s, _, _ in together])
    b.run([acc[:steps] for _, acc, steps in together])
    for (s1, _, steps), (s2, _, _) in zip(alone, together):
        assert s1.t == s2.t
        assert np.array_equal(s1.listeners(), s2.listeners())
        for rel in (0, -1, -2):
            assert np.array_equal(s1.grid(rel), s2.grid(rel))
        assert np.array_equal(s1.dump("dirichlet"), s2.dump("dirichlet"))
    # both sides continue one by one: the batch left every scene's state consistent
    for (s1, acc, steps), (s2, _, _) in zip(alone, together):
        s1.step(acc[steps: steps + 30])
        s2.step(acc[steps: steps + 30])
        assert np.array_equal(s1.listeners(), s2.listeners())
    # a second batch run on the continued scenes, device accelerations
    import torch

    more = [torch.from_numpy(sine_acc(19, s.nt, 700.0, 1e-5)).cuda() for s, _, _ in together]
    for (s1, _, _), a in zip(alone, more):
        s1.step(a)
    b.run(more)
    torch.cuda.synchronize()
    for (s1, _, _), (s2, _, _) in zip(alone, together):
        assert np.array_equal(s1.listeners(), s2.listeners())
    b.close()
    for s, _, _ in alone + together:
        s.close()


def test_batch_rejects_bad_sets(gpu):
    s, f, dt = _scene(20, 1, 9)
    with pytest.raises(PPPMError):
        Batch([s, s])
    p, _, _ = _scene(24, 1, 10, pml_width=3)
    with pytest.raises(PPPMError):
        Batch([s, p])
    s.close()
    p.close()


def test_batch_with_motion_frames_matches_single_scenes(gpu):
    """Moving scenes in a batch: every motion frame updates each scene's mesh
    (PPPMSolver::update_mesh, pppm.h:98-110), then one batch run advances all scenes through the
    frame's steps.  Lists, caches and corrected-cell counts change from frame to frame; the
    listener series and fields stay bit-identical to stepping each scene alone with the same
    frames, and the batch's recorded graphs are reused across frames."""
    from helpers import moving_small_verts

    specs = [(24, 2, 21, 1100.0), (20, 1, 22, 900.0), (28, 2, 23, 1300.0)]
    every, frames = 12, 8

    def make():
        out = []
        for res, sub, seed, fq in specs:
            s, f, dt = _scene(res, sub, seed)
            out.append((s, f, dt, fq))
        return out

    def verts_of(res, sub, seed, step, dt):
        rng = np.random.default_rng(seed)
        v, _ = scenes.icosphere(sub)
        v = v * (1 + 0.08 * rng.uniform(-1, 1, (len(v), 1)))
        v = (v * 0.1).astype(np.float32)
        return moving_small_verts(v, step, dt)

    alone, together = make(), make()
    b = Batch([s for s, _, _, _ in together])
    for fr in range(frames):
        rows = []
        for (res, sub, seed, _), (s1, f, dt, fq), (s2, _, _, _) in zip(specs, alone, together):
            if fr:
                v = verts_of(res, sub, seed, fr * every, dt)
                s1.update_mesh(v)
                s2.update_mesh(v)
            a = sine_acc(every, len(f), fq, dt, first=fr * every)
            s1.step(a)
            rows.append(a)
        b.run(rows)
    for (s1, _, _, _), (s2, _, _, _) in zip(alone, together):
        assert s1.t == s2.t
        assert np.array_equal(s1.listeners(), s2.listeners())
        assert np.all(np.isfinite(s1.listeners()))
        for rel in (0, -1):
            assert np.array_equal(s1.grid(rel), s2.grid(rel))
    b.close()
    for s, _, _, _ in alone + together:
        s.close()


def test_batch_with_a_scene_near_the_boundary(gpu):
    """A scene whose mesh reaches cell 3 of an axis steps unsplit (its corrected cells neighbour the
    boundary layer); a batch holding it records the unsplit stencil for every scene, with results
    bit-identical to the scenes stepped one by one."""
    def make():
        v, f, h, mn, dt = edge_sphere(0, 3)
        e = Solver(24, h, dt, mn)
        e.set_mesh(v, f)
        e.add_listener(20, 12, 12)
        e.add_listener(1, 12, 12)
        s, f2, dt2 = _scene(24, 2, 2)
        return [(e, sine_acc(80, len(f), 1500.0, dt), 61), (s, sine_acc(80, len(f2), 1100.0, dt2), 45)]

    alone = make()
    for s, acc, steps in alone:
        s.step(acc[:steps])
    together = make()
    b = Batch([s for s, _, _ in together])
    b.run([acc[:steps] for _, acc, steps in together])
    for (s1, acc, steps), (s2, _, _) in zip(alone, together):
        assert np.array_equal(s1.listeners(), s2.listeners())
        for rel in (0, -1, -2):
            assert np.array_equal(s1.grid(rel), s2.grid(rel))
        s1.step(acc[steps:])
        s2.step(acc[steps:])
        assert np.array_equal(s1.listeners(), s2.listeners())
    b.close()
    for s, _, _ in alone + together:
        s.close()
