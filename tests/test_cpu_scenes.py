"""Host-side scene generation (pppm_b200.scenes) on the CPU: the large moving scene stays inside the
reference's fixed list capacities and keeps its two bodies apart, its band-limited noise is
reproducible whatever step ranges are asked for, and motion frames split the steps without gaps."""
import math

import numpy as np
import pytest

from pppm_b200 import scenes


def _max_block_count(centres, min_pos, h, lo, hi, base=False):
    """Largest number of triangle centres in a (hi - lo)^3 block of cells around any occupied cell
    (3^3 around each triangle's cell, or 4^3 from base - 1 .. base + 2 around each base cell)."""
    g = (centres - min_pos) / h
    cell = np.floor(g - 0.5 if base else g).astype(np.int64)
    own = np.floor(g).astype(np.int64)
    counts = {}
    for c in map(tuple, own):
        counts[c] = counts.get(c, 0) + 1
    best = 0
    for c in set(map(tuple, cell)):
        n = 0
        for dx in range(lo, hi):
            for dy in range(lo, hi):
                for dz in range(lo, hi):
                    n += counts.get((c[0] + dx, c[1] + dy, c[2] + dz), 0)
        best = max(best, n)
    return best


@pytest.fixture(scope="module")
def large():
    return scenes.LargeScene()


def test_large_scene_shape(large):
    assert large.res == 128
    assert len(large.tris) == 2 * 20480
    assert large.nv == 2 * 10242
    assert large.tris.min() == 0 and large.tris.max() == large.nv - 1
    # frames: dt from the demo driver's rule, 1 kHz motion frames of ~82 steps
    r = scenes.frame_ranges(large, 3)
    assert r[0][0] == 0 and all(a[1] == b[0] for a, b in zip(r, r[1:]))
    assert all(80 <= b - a <= 84 for a, b in r)


@pytest.mark.parametrize("frame", [0, 61, 173, 244])
def test_large_scene_within_reference_capacities(large, frame):
    # the reference's fixed list sizes (particle_grid.h:9-11): 3^3 lists <= 256, 4^3 <= 512
    v = large.frame_verts(frame).astype(np.float64)
    c = v[large.tris].mean(1)
    assert _max_block_count(c, large.min_pos, large.h, -1, 2) < 256
    assert _max_block_count(c, large.min_pos, large.h, -1, 3, base=True) < 512
    # every vertex inside the grid, away from the absorbing layers
    g = (v - large.min_pos) / large.h
    assert g.min() > 3 and g.max() < large.res - 3


@pytest.mark.parametrize("frame", [0, 100, 244])
def test_large_scene_bodies_stay_apart(large, frame):
    # more than 4 cells between the spheres: no face pair joins them
    v = large.frame_verts(frame)
    a, b = v[: large.nv // 2].astype(np.float64), v[large.nv // 2:].astype(np.float64)
    gap = np.linalg.norm(a.mean(0) - b.mean(0)) - np.linalg.norm(a - a.mean(0), axis=1).max() \
        - np.linalg.norm(b - b.mean(0), axis=1).max()
    assert gap > 4 * large.h


def test_streamed_noise_reproducible_and_band_limited():
    dt = 1.0 / 80000
    n1 = scenes.StreamedNoise(6, dt, 100.0, 8000.0, seed=5)
    n2 = scenes.StreamedNoise(6, dt, 100.0, 8000.0, seed=5)
    full = n1.get(0, 4096)
    # any range, in any order, gives the same values
    assert np.array_equal(n2.get(1000, 300), full[:, 1000:1300])
    assert np.array_equal(n2.get(5, 17), full[:, 5:22])
    assert np.array_equal(n2.get(4000, 96), full[:, 4000:4096])
    # unit RMS (within sampling error) and little energy outside the band
    x = full[:, 512:]
    assert 0.85 < float(np.sqrt((x.astype(np.float64) ** 2).mean())) < 1.15
    X = np.abs(np.fft.rfft(x, axis=1)) ** 2
    f = np.fft.rfftfreq(x.shape[1], dt)
    outside = X[:, (f < 30.0) | (f > 16000.0)].sum() / X.sum()
    assert outside < 0.02
    # a different seed gives different noise
    n3 = scenes.StreamedNoise(6, dt, 100.0, 8000.0, seed=6)
    assert not np.allclose(n3.get(0, 512), full[:, :512])


def test_large_scene_accelerations(large):
    a = large.acc(100, 3)
    assert a.shape == (3, len(large.tris)) and a.dtype == np.float32
    assert np.all(np.isfinite(a))
    # per-vertex noise averaged to triangles: both bodies carry it
    assert np.abs(a[:, :20480]).mean() > 0.1 and np.abs(a[:, 20480:]).mean() > 0.1


def test_frame_ranges_match_frame_of_step():
    sc = scenes.MovingScene()
    r = scenes.frame_ranges(sc, 5)
    for f, (a, b) in enumerate(r):
        assert all(sc.frame_of_step(s) == f for s in range(a, b))
        assert sc.frame_of_step(b) == f + 1
    assert math.isclose(sc.frame_hz, 1000.0)
