"""The CPU oracle pinned against the reference's own test suite (run on the CPU).

Each test restates one reference test (file cited) on seeded inputs:
  tests/ParticleGridTest.cu:10-235   triangle records, per-cell binning, 3^3 / 4^3 lists after
                                     random moves (counts exact, membership by position)
  tests/FaceCacheTest.cu:27-72       interpolation weights reproduce the 1-point integral of a
                                     trilinear function (margin J * 1e-5)
  tests/TDBEMTest.cu:8-70            time-domain weights against the frequency-domain
                                     (Helmholtz) response at steady state (10 %)
  tests/GridCacheTest.cu:16-64       cached FDTD-near / BEM-near weights against the direct
                                     per-target evaluation of pppm_direct.h:15-58
"""
import numpy as np
import pytest

from oracle import oracle as O


def random_scene(n, res=64, seed=0, h=0.005):
    """random_pppm of tests/case_generator.h:29-50: small random right triangles of size ~h
    placed in the interior, with our own seeded generator."""
    rng = np.random.default_rng(seed)
    v = np.zeros((3 * n, 3), np.float32)
    f = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    for i in range(n):
        sgn = rng.choice([-1.0, 1.0], size=3)
        off = rng.uniform(0, 1, 3) * (res - 8) * h + 4 * h
        v[3 * i] = np.array([0, 0, 1.0]) * rng.uniform() * sgn[0] * h + off
        v[3 * i + 1] = np.array([1.0, 0, 0]) * rng.uniform() * sgn[1] * h + off
        v[3 * i + 2] = np.array([0, 1.0, 0]) * rng.uniform() * sgn[2] * h + off
    return v, f


def cell_center(x, y, z, h, mn=(0, 0, 0)):
    return np.array([(x + 0.5) * h + mn[0], (y + 0.5) * h + mn[1], (z + 0.5) * h + mn[2]], np.float32)


def test_particle_grid_invariants():
    res, h, dt = 64, np.float32(0.005), np.float32(8e-6)
    v, f = random_scene(1024, res)
    o = O.Oracle(res, h, dt)
    o.set_mesh(v, f)
    rng = np.random.default_rng(1)
    for _ in range(5):
        v = v + (rng.uniform(0, 1, v.shape) * h * 0.1).astype(np.float32)
        o.update_mesh(v)
    geom, cells = o.triangles()
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    cr = np.cross(b - a, c - a)
    np.testing.assert_allclose(geom[:, 6], 0.5 * np.linalg.norm(cr, axis=1), rtol=1e-3)
    np.testing.assert_allclose(geom[:, 3:6], cr / np.linalg.norm(cr, axis=1)[:, None], rtol=1e-3, atol=1e-6)
    np.testing.assert_allclose(geom[:, :3], (a + b + c) / 3, rtol=1e-3)
    L = o.lists()
    cc = L["cell_counts"].reshape((res,) * 3)
    assert cc.sum() == len(f)
    # every triangle sits in its cell, and its base cell spans its centre
    for i in range(len(f)):
        ctr = geom[i, :3]
        cen = cell_center(*cells[i, :3], h)
        assert np.all(ctr >= cen - h / 2) and np.all(ctr < cen + h / 2 + 1e-7)
        base = cell_center(*cells[i, 3:], h)
        assert np.all(ctr >= base - 1e-7) and np.all(ctr < base + h + 1e-7)
    # 3^3 lists: every inner cell with a non-empty block, counts equal to the block sum,
    # members within 1.5 h of the cell centre
    pad = np.pad(cc, 1)
    block3 = sum(pad[1 + dx: 1 + dx + res, 1 + dy: 1 + dy + res, 1 + dz: 1 + dz + res]
                 for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1))
    inner = np.zeros_like(block3, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    assert len(L["n3_cells"]) == int(((block3 > 0) & inner).sum())
    o3 = 0
    for x, y, z, n in L["n3_cells"]:
        assert n == block3[x, y, z]
        tris = L["n3_tris"][o3: o3 + n]
        o3 += n
        d = np.abs(geom[tris, :3] - cell_center(x, y, z, h))
        assert np.all(d < 1.5 * h + 1e-7)
    # 4^3 lists of non-empty base cells
    o4 = 0
    for x, y, z, nb in L["b4_cells"]:
        n = int(cc[x - 1: x + 3, y - 1: y + 3, z - 1: z + 3].sum())
        tris = L["n4_tris"][o4: o4 + n]
        o4 += n
        d = geom[tris, :3] - cell_center(x, y, z, h)
        assert np.all(d >= -1.5 * h - 1e-7) and np.all(d < 2.5 * h + 1e-7)
    assert o4 == len(L["n4_tris"])
    o.close()


def test_interpolation_weights_reproduce_trilinear_functions():
    res, h, dt = 32, np.float32(0.005), np.float32(8e-6)
    v, f = random_scene(512, res, seed=3)
    o = O.Oracle(res, h, dt)
    o.set_mesh(v, f)
    w = o.interp()
    _, cells = o.triangles()
    rng = np.random.default_rng(4)
    p = rng.uniform(size=8)

    def func(x):  # trilinear in the cell-normalised coordinates
        x, y, z = x / h
        return p[0] * x + p[1] * y + p[2] * z + p[3] * x * y + p[4] * x * z + p[5] * y * z + p[6] * x * y * z + p[7]

    for i in range(len(f)):
        val = 0.0
        for j in range(8):
            q = cells[i, 3:] + np.array([(j >> 2) & 1, (j >> 1) & 1, j & 1])
            val += func(cell_center(*q, h).astype(np.float64)) * w[i, j]
        a, b, c = v[f[i]].astype(np.float64)
        jac = np.linalg.norm(np.cross(b - a, c - a))
        truth = 0.5 * jac * func((a + b + c) / 3)
        assert abs(val - truth) <= jac * 1e-5 * max(1.0, abs(truth / jac))
    o.close()


@pytest.mark.parametrize("to_point", [True, False])
def test_tdbem_time_domain_matches_helmholtz(to_point):
    rng = np.random.default_rng(7 if to_point else 8)
    scale = 0.01
    V = (rng.uniform(size=(6, 3)) * scale).astype(np.float32)
    src, trg = [0, 1, 2], [3, 4, 5]
    pt = (rng.uniform(size=3) * scale).astype(np.float32)
    c = 340.3
    for trial in range(3):
        dt = np.float32(rng.integers(100, 201) * 1e-7)
        freq = float(rng.integers(1000, 4001))
        om = 2 * np.pi * freq
        w = O.laplace_weight(dt, 0.01, V.ravel(), src, point=pt if to_point else None,
                             face=None if to_point else trg)
        S, D = O.pair_integral(0.01, V.ravel(), src, om / c, point=pt if to_point else None,
                               face=None if to_point else trg)
        na, da = rng.uniform(), rng.uniform()
        t = np.arange(-16, 16)
        N = np.cos(om * t * float(dt)) * na
        Dh = np.cos(om * t * float(dt)) * da
        lap = np.array([sum(-w[k] * N[16 + tt - k] + w[16 + k] * Dh[16 + tt - k] for k in range(16))
                        for tt in range(16)])
        hw = -S * na + D * da
        helm = np.array([(hw * np.exp(1j * om * tt * float(dt))).real for tt in range(16)])
        amp = np.abs(hw)
        assert np.max(np.abs(lap - helm)) / amp < 0.1


def test_grid_cache_equals_direct_evaluation():
    """Cached FDTD-near / BEM-near weights (pppm_cache.cu:64-123) equal the direct per-target
    sums of pppm_direct.h:15-58: for a source triangle and destination cell c,
    far correction = 2 near(c, t-1) + s (sum_{+-e} near(c +- e) - 6 near(c))(t-1) - near(c, t-2),
    sources inside the destination cell skipped."""
    res, h, dt = 16, np.float32(0.005), np.float32(8e-6)
    v, f = random_scene(12, res, seed=5)
    o = O.Oracle(res, h, dt, precision="fp64")
    o.set_mesh(v, f)
    gw = o.grid_weights()
    _, cells = o.triangles()
    s = (340.3 * float(dt) / float(h)) ** 2
    for tri in range(0, len(f), 3):
        tc = cells[tri, :3]
        for woff in (0, 4, 13, 22, 26):
            nb = tc + np.array([woff % 3 - 1, woff // 3 % 3 - 1, woff // 9 - 1])

            def w_at(q):
                if np.all(q == tc):
                    return np.zeros(32)
                return O.laplace_weight(dt, h, v.ravel(), f[tri], point=cell_center(*q, h))

            w0 = w_at(nb)
            lap = sum(w_at(nb + e) for e in np.vstack([np.eye(3, dtype=int), -np.eye(3, dtype=int)])) - 6 * w0
            one = 2 * w0 + s * lap  # applied one step back
            exp_f = np.zeros(32)
            for half in (0, 16):
                exp_f[half + 1: half + 16] += one[half: half + 15]
                exp_f[half + 2: half + 16] -= w0[half: half + 14]
            got_f, got_b = gw[tri, woff], gw[tri, 27 + woff]
            for half in (slice(0, 16), slice(16, 32)):
                sc = max(np.abs(exp_f[half]).max(), 1e-30)
                assert np.abs(got_f[half] - exp_f[half]).max() / sc < 1e-5
                sc = max(np.abs(w0[half]).max(), 1e-30)
                assert np.abs(got_b[half] - w0[half]).max() / sc < 1e-5
    o.close()


def test_oracle_fp32_step_close_to_fp64_step():
    """The two precisions of the same scheme stay close over a short run (fp16 weight storage
    is the dominant difference)."""
    from pppm_b200 import scenes

    v, f = scenes.icosphere(2)
    v = (v * 0.1).astype(np.float32)
    res = 24
    h, mn = scenes.grid_for_bbox(v.min(0), v.max(0), res, 2.0)
    dt = np.float32(0.5 * h / (np.sqrt(3) * 340.3))
    acc = np.repeat(np.sin(2 * np.pi * 1500 * np.arange(150) * float(dt)).astype(np.float32)[:, None], len(f), 1)
    out = {}
    for prec in ("fp32", "fp64"):
        o = O.Oracle(res, h, dt, mn, precision=prec)
        o.set_mesh(v, f)
        out[prec] = o.step(acc, listeners=[(20, 20, 20)])[:, 0]
        o.close()
    err = np.linalg.norm(out["fp32"] - out["fp64"]) / np.linalg.norm(out["fp64"])
    assert err < 5e-3
