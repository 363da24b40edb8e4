"""Shared scene builders and comparison helpers for the tests."""
import os

import numpy as np

from pppm_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# Grid offset (in cells) that keeps the symmetric icosphere's triangle centres off cell faces:
# centred grids put many centres exactly on a face, where the device's approximate division
# and the CPU oracle's IEEE division may round to neighbouring cells.
OFFSET = np.array([0.137, 0.291, 0.0713])


def sphere_small(res=24, sub=2, radius=0.1, offset=True):
    v, f = scenes.icosphere(sub)
    v = (v * radius).astype(np.float32)
    h, mn = scenes.grid_for_bbox(v.min(0), v.max(0), res, 2.0)
    if offset:
        mn = (mn + OFFSET * h).astype(np.float32)
    dt = np.float32(0.5 * h / (np.sqrt(3) * 340.3))
    return v, f, h, mn, dt


def moving_small_verts(v0, step, dt):
    t = step * float(dt)
    R = scenes.rotation_matrix([0.3, 0.5, 0.8], 40.0 * t)
    v = v0.astype(np.float64) @ R.T
    v[:, 0] += 0.01 * np.sin(2 * np.pi * 60.0 * t)
    return v.astype(np.float32)


def sine_acc(steps, nt, freq, dt, first=0):
    a = np.sin(2 * np.pi * freq * (np.arange(first, first + steps) * float(dt))).astype(np.float32)
    return np.repeat(a[:, None], nt, 1)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def per_cell_sets(cells, tris):
    """{(x, y, z): sorted tuple of triangle ids} from a (n, 4) cell table and concatenated lists."""
    out, o = {}, 0
    for x, y, z, n in cells:
        out[(int(x), int(y), int(z))] = tuple(sorted(int(t) for t in tris[o: o + n]))
        o += n
    return out


def records_to_taps(rec):
    """72-byte fp16 records -> (n, 32) float32 taps (single 16 then double 16) as the reference
    convolution reads them, (float)half * scale (bem.h:203-213)."""
    s = rec["s"].astype(np.float32) * rec["ms"][:, None]
    d = rec["d"].astype(np.float32) * rec["md"][:, None]
    return np.concatenate([s, d], 1)


def golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        return None
    return dict(np.load(path, allow_pickle=False))


def reference_noise_floor(name, steps=None):
    """Largest relative L2 difference between the reference's own runs of one scene (the golden
    series and the repeats in noise.npz, listener 0).  The reference accumulates its correction
    sums with float atomics, so its repeats differ; the scheme amplifies that rounding step by
    step, and agreement with it is only meaningful up to this floor."""
    g, n = golden(name + ".npz"), golden("noise.npz")
    if g is None or n is None or name not in n:
        return None
    runs = [g["series"][:, 0]] + list(n[name])
    if steps is not None:
        runs = [r[:steps] for r in runs]
    return max(rel_l2(runs[i], runs[j]) for i in range(len(runs)) for j in range(i + 1, len(runs)))
