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


def edge_sphere(axis, cell):
    """sphere_small moved along one axis so that its triangles' cells reach `cell` there at one end
    (the lowest cell when cell < 12, else the highest)"""
    v0, f, h, mn, dt = sphere_small()
    c = v0[f].mean(1)
    rel = (c[:, axis] - mn[axis]) / h
    shift = (cell + 0.5 - rel.min()) if cell < 12 else (cell + 0.5 - rel.max())
    v = v0.copy()
    v[:, axis] += np.float32(shift * h)
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


def dyadic(rng, shape, bits=10):
    """standard normal samples rounded to multiples of 2^-bits (float32): x + eps v and x - eps v
    are then exact in float32 for eps = 2^-3, so a central difference is taken about x itself"""
    return (np.round(rng.standard_normal(shape) * 2.0 ** bits) / 2.0 ** bits).astype(np.float32)


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


def cell_list_codes(cells, tris, res, nt):
    """Sorted int64 codes (linear cell index * nt + triangle) of per-cell lists given as a (n, 4)
    table (x, y, z, list length) and the concatenated lists: equal arrays <=> equal lists as sets
    per cell, compared without a Python loop (whole-run tests compare them every motion frame)."""
    cells = np.asarray(cells, np.int64).reshape(-1, 4)
    lin = (cells[:, 0] * res + cells[:, 1]) * res + cells[:, 2]
    own = np.repeat(lin, cells[:, 3])
    t = np.asarray(tris, np.int64)[: len(own)]
    return np.sort(own * nt + t)


def window_counts(cell_counts, res, cells, lo=1, hi=2):
    """Sum of per-cell triangle counts over the box [x - lo, x + hi]^3 (clipped to the grid) of
    each (x, y, z) row: the 4^3 list length of a base cell (particle_grid.cu: neighbours -1..+2)."""
    c = np.asarray(cell_counts, np.int64).reshape((res,) * 3)
    s = np.zeros((res + 1,) * 3, np.int64)
    s[1:, 1:, 1:] = c.cumsum(0).cumsum(1).cumsum(2)
    cells = np.asarray(cells, np.int64).reshape(-1, 4)
    a = np.clip(cells[:, :3] - lo, 0, res)
    b = np.clip(cells[:, :3] + hi + 1, 0, res)
    x0, y0, z0 = a.T
    x1, y1, z1 = b.T
    return (s[x1, y1, z1] - s[x0, y1, z1] - s[x1, y0, z1] - s[x1, y1, z0] + s[x0, y0, z1] + s[x0, y1, z0] +
            s[x1, y0, z0] - s[x0, y0, z0])


def face_pair_codes(b4_cells, b4_tris, n4_tris, n4_len, nt):
    """Sorted int64 codes (centre * nt + neighbour) of the face pairs that base cells define:
    every centre triangle of a base cell against every triangle of that cell's 4^3 list."""
    b4 = np.asarray(b4_cells, np.int64).reshape(-1, 4)
    nb = b4[:, 3]
    n4_len = np.asarray(n4_len, np.int64)
    cb = np.concatenate([[0], np.cumsum(nb)])
    c4 = np.concatenate([[0], np.cumsum(n4_len)])
    bt = np.asarray(b4_tris, np.int64)
    l4 = np.asarray(n4_tris, np.int64)
    out = []
    for i in range(len(b4)):
        if nb[i] and n4_len[i]:
            cen = bt[cb[i]: cb[i + 1]]
            lst = l4[c4[i]: c4[i + 1]]
            out.append((cen[:, None] * nt + lst[None, :]).ravel())
    return np.sort(np.concatenate(out)) if out else np.zeros(0, np.int64)


def point_triangle_distance(p, a, b, c):
    """Euclidean distance (float64) from points p (n, 3) to triangles (a, b, c) (n, 3 each)."""
    return np.linalg.norm(p - closest_point_on_triangle(p, a, b, c), axis=1)


def closest_point_on_triangle(p, a, b, c):
    """Closest points (float64) of triangles (a, b, c) (n, 3 each) to points p (n, 3), by the
    Voronoi-region construction (Ericson, Real-Time Collision Detection 5.1.5)."""
    p, a, b, c = (np.asarray(x, np.float64) for x in (p, a, b, c))
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = (ab * ap).sum(1), (ac * ap).sum(1)
    bp = p - b
    d3, d4 = (ab * bp).sum(1), (ac * bp).sum(1)
    cp = p - c
    d5, d6 = (ab * cp).sum(1), (ac * cp).sum(1)
    va = d3 * d6 - d5 * d4
    vb = d5 * d2 - d1 * d6
    vc = d1 * d4 - d3 * d2
    q = np.empty_like(p)
    done = np.zeros(len(p), bool)

    def put(mask, val):
        m = mask & ~done
        q[m] = val[m] if val.ndim == 2 else val
        done[m] = True

    put((d1 <= 0) & (d2 <= 0), a)
    put((d3 >= 0) & (d4 <= d3), b)
    with np.errstate(divide="ignore", invalid="ignore"):
        v = d1 / (d1 - d3)
        put((vc <= 0) & (d1 >= 0) & (d3 <= 0), a + v[:, None] * ab)
        put((d6 >= 0) & (d5 <= d6), c)
        w = d2 / (d2 - d6)
        put((vb <= 0) & (d2 >= 0) & (d6 <= 0), a + w[:, None] * ac)
        w2 = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        put((va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0), b + w2[:, None] * (c - b))
        den = 1.0 / (va + vb + vc)
        v2, w3 = vb * den, vc * den
        put(np.ones(len(p), bool), a + v2[:, None] * ab + w3[:, None] * ac)
    return q
