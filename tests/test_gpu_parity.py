"""libpppm_b200 (CUDA, through the C ABI) against the CPU oracle on identical seeded inputs.

Tolerances:
  integer structures (lists, labels)       bit-exact (lists compared as per-cell sets)
  FDTD + absorbing boundary / PML fields    max |diff| <= 1e-5 of the field scale (the
                                            device boundary solve uses fused multiply-adds and
                                            approximate division like the reference; the oracle
                                            is IEEE C)
  listener series (FP32 scheme)             relative L2 <= 1e-5 over the first 50 steps and
                                            <= 1e-3 over 300 steps: the scheme amplifies
                                            rounding differences step after step (summing the
                                            same pairs in reverse order moves a 300-step series
                                            by ~3e-5), and the device sums in another order
                                            with fused multiply-adds
  TDBEM weights vs the FP64 oracle          |diff| <= 5e-3 of the row's max-abs scale (FP32
                                            fast-math evaluation + fp16 storage vs FP64)
  nearest-triangle indices                  may differ where two triangles are equally near
                                            (last-ulp distance differences decide the tie); the
                                            distances themselves must agree
"""
import numpy as np
import pytest

from helpers import moving_small_verts, per_cell_sets, records_to_taps, rel_l2, sine_acc, sphere_small
from oracle.oracle import Oracle
from pppm_b200 import Solver, scenes

pytestmark = pytest.mark.gpu


def _impulse(res, rng):
    g = np.zeros((res,) * 3, np.float32)
    g[res // 2, res // 2, res // 2] = 1.0
    g[res // 3: res // 3 + 5, res // 2 - 2: res // 2 + 2, res // 2: res // 2 + 2] += rng.uniform(
        -0.1, 0.1, size=(5, 4, 2)).astype(np.float32)
    return g


@pytest.mark.parametrize("pml", [0, 3])
def test_fdtd_impulse_matches_oracle(gpu, pml):
    rng = np.random.default_rng(1)
    res, dl = 20, 0.01
    dt = np.float32(0.5 * dl / (np.sqrt(3) * 340.3))
    g0 = _impulse(res, rng)
    s = Solver(res, dl, dt, pml_width=pml)
    o = Oracle(res, dl, dt, pml_width=pml)
    s.t = 0
    o.t = 0
    for x in (s,):
        x.load("grid_t", g0)
        x.load("grid_tm1", 0.5 * g0)
    o.write_grid(0, g0)
    o.write_grid(-1, 0.5 * g0)
    s.step(None, nsteps=60)
    o.step(None, nsteps=60)
    assert s.t == o.t == 60
    for rel in (0, -1):
        a, b = s.grid(rel), o.grid(rel)
        scale = np.abs(b).max()
        assert np.abs(a - b).max() <= 1e-5 * scale, (rel, np.abs(a - b).max(), scale)
    s.close()


def _static_pair(res=24):
    v, f, h, mn, dt = sphere_small(res)
    s = Solver(res, h, dt, mn)
    o = Oracle(res, h, dt, mn)
    s.set_mesh(v, f)
    o.set_mesh(v, f)
    return s, o, v, f, h, mn, dt


def test_lists_bit_exact(gpu):
    s, o, v, f, *_ = _static_pair()
    Lo = o.lists()
    assert np.array_equal(s.dump("cell_counts"), Lo["cell_counts"])
    assert np.array_equal(s.dump("n3_cells").reshape(-1, 4), Lo["n3_cells"])
    assert np.array_equal(s.dump("n3_tris"), Lo["n3_tris"])
    assert np.array_equal(s.dump("b4_cells").reshape(-1, 4), Lo["b4_cells"])
    assert np.array_equal(s.dump("n4_tris"), Lo["n4_tris"])
    assert np.array_equal(s.dump("face_pairs").reshape(-1, 2), o.face_pairs())
    gs, cs = s.dump("tri_geom").reshape(-1, 7), s.dump("tri_cells").reshape(-1, 6)
    go, co = o.triangles()
    assert np.array_equal(cs, co)
    np.testing.assert_allclose(gs, go, rtol=1e-5, atol=1e-7)
    s.close()


def test_weights_close_to_fp64_oracle(gpu):
    s, o, *_ = _static_pair()
    wg = records_to_taps(s.dump("grid_cache"))
    wo = o.grid_weights().reshape(-1, 32)
    for half in (slice(0, 16), slice(16, 32)):
        scale = np.maximum(np.abs(wo[:, half]).max(1, keepdims=True), 1e-30)
        err = np.abs(wg[:, half] - wo[:, half]) / scale
        assert err.max() < 5e-3, err.max()
    wf = records_to_taps(s.dump("face_cache"))
    wfo = o.face_weights()
    for half in (slice(0, 16), slice(16, 32)):
        scale = np.maximum(np.abs(wfo[:, half]).max(1, keepdims=True), 1e-30)
        err = np.abs(wf[:, half] - wfo[:, half]) / scale
        assert err.max() < 5e-3, err.max()
    np.testing.assert_allclose(s.dump("interp").reshape(-1, 8), o.interp(), rtol=1e-5, atol=1e-9)
    s.close()


def test_static_step_matches_oracle_with_shared_tables(gpu):
    s, o, v, f, h, mn, dt = _static_pair()
    # the oracle runs the reference's step order with the GPU's own tables
    o.import_grid_cache(s.dump("grid_cache"))
    o.import_face_cache(s.dump("face_pairs").reshape(-1, 2), s.dump("face_cache"))
    listeners = [(20, 20, 20), (12, 12, 17)]
    for lx in listeners:
        s.add_listener(*lx)
    acc = sine_acc(300, len(f), 1500.0, dt)
    s.step(acc)
    ref = o.step(acc, listeners=listeners)
    got = s.listeners()
    assert got.shape == ref.shape
    for l in range(len(listeners)):
        assert rel_l2(got[:50, l], ref[:50, l]) < 1e-5, rel_l2(got[:50, l], ref[:50, l])
        assert rel_l2(got[:, l], ref[:, l]) < 1e-3, rel_l2(got[:, l], ref[:, l])
    assert rel_l2(s.grid(0), o.grid(0)) < 1e-3
    n_s, d_s = s.dump("neumann").reshape(-1, 32), s.dump("dirichlet").reshape(-1, 32)
    n_o, d_o = o.history()
    assert np.array_equal(n_s, n_o)
    assert rel_l2(d_s, d_o) < 1e-3
    s.close()


def test_moving_mesh_lists_and_series(gpu):
    v0, f, h, mn, dt = sphere_small()
    res = 24
    s, o = Solver(res, h, dt, mn), Oracle(res, h, dt, mn)
    s.set_mesh(moving_small_verts(v0, 0, dt), f)
    o.set_mesh(moving_small_verts(v0, 0, dt), f)
    s.add_listener(20, 20, 20)
    acc = sine_acc(120, len(f), 1200.0, dt)
    ref = []
    for s0 in range(0, 120, 10):
        if s0:
            vv = moving_small_verts(v0, s0, dt)
            s.update_mesh(vv)
            o.update_mesh(vv)
            Lo = o.lists()
            assert np.array_equal(s.dump("n3_tris"), Lo["n3_tris"])
            assert np.array_equal(s.dump("n4_tris"), Lo["n4_tris"])
        # share tables so the comparison isolates the step and the cache bookkeeping
        o.import_grid_cache(s.dump("grid_cache"))
        o.import_face_cache(s.dump("face_pairs").reshape(-1, 2), s.dump("face_cache"))
        s.step(acc[s0: s0 + 10])
        ref.append(o.step(acc[s0: s0 + 10], listeners=[(20, 20, 20)]))
    got, want = s.listeners()[:, 0], np.concatenate(ref)[:, 0]
    assert rel_l2(got[:50], want[:50]) < 1e-5
    assert rel_l2(got, want) < 1e-3
    s.close()


def test_fp64_scheme_matches_fp64_oracle(gpu):
    v, f, h, mn, dt = sphere_small()
    res = 24
    s = Solver(res, h, dt, mn, precision="fp64")
    o = Oracle(res, h, dt, mn, precision="fp64")
    s.set_mesh(v, f)
    o.set_mesh(v, f)
    s.add_listener(20, 20, 20)
    acc = sine_acc(200, len(f), 1500.0, dt)
    s.step(acc)
    ref = o.step(acc, listeners=[(20, 20, 20)])
    assert rel_l2(s.listeners()[:, 0], ref[:, 0]) < 1e-7
    s.close()


def test_fp32_vs_fp64_error_small(gpu):
    v, f, h, mn, dt = sphere_small()
    res = 24
    out = {}
    for prec in ("fp32", "fp64"):
        s = Solver(res, h, dt, mn, precision=prec)
        s.set_mesh(v, f)
        s.add_listener(20, 20, 20)
        s.step(sine_acc(300, len(f), 1500.0, dt))
        out[prec] = s.listeners()[:, 0]
        s.close()
    assert rel_l2(out["fp32"], out["fp64"]) < 5e-3


def test_cell_labels_match_oracle(gpu):
    v, f, h, mn, dt = sphere_small()
    res = 24
    s, o = Solver(res, h, dt, mn), Oracle(res, h, dt, mn)
    s.set_mesh(v, f)
    o.set_mesh(v, f)
    g = s.classify_cells()
    ref = o.classify()
    assert np.array_equal(s.dump("cell_type"), ref["type"])
    assert np.array_equal(s.dump("cell_ghost"), ref["ghost"])
    assert g == ref["ghost_count"]
    same = s.dump("cell_nearest") == ref["nearest"]
    assert same.mean() > 0.95
    pts = s.dump("cell_points").reshape(-1, 7)
    np.testing.assert_allclose(pts[~same, 6], ref["points"][~same, 6], rtol=1e-5)
    s.close()


def test_fresh_cells_match_oracle(gpu):
    rng = np.random.default_rng(5)
    v, f, h, mn, dt = sphere_small()
    res = 24
    s, o = Solver(res, h, dt, mn), Oracle(res, h, dt, mn)
    s.set_mesh(v, f)
    o.set_mesh(v, f)
    s.classify_cells()
    o.classify()
    g_t = rng.uniform(-1, 1, (res,) * 3).astype(np.float32)
    g_tm1 = rng.uniform(-1, 1, (res,) * 3).astype(np.float32)
    s.load("grid_t", g_t)
    s.load("grid_tm1", g_tm1)
    o.write_grid(0, g_t)
    o.write_grid(-1, g_tm1)
    v1 = v.copy()
    v1[:, 0] += 1.3 * h
    s.update_mesh(v1)
    o.update_mesh(v1)
    # uniform accelerations: where two triangles tie for nearest the fill is the same either way
    a0 = np.full(len(f), -0.3, np.float32)
    a1 = np.full(len(f), 0.7, np.float32)
    n = s.fill_fresh_cells(a1, a0)
    cls = o.classify()
    m = o.fresh(a1, a0)
    assert n == m and n > 0
    # Two ties are decided by last-ulp rounding (device fast-math vs the oracle's IEEE C):
    # two triangles equally near a cell, and a reflection point lying on a plane of cell
    # centres (the 8 interpolation cells then shift by one).  The other cells must agree to
    # tolerance; the ties must stay few.
    same = (s.dump("cell_nearest") == cls["nearest"]).ravel()
    pts = cls["points"].reshape(-1, 7)
    idx = np.arange(res ** 3)
    ijk = np.stack([idx // (res * res), (idx // res) % res, idx % res], 1)
    xf = (ijk + 0.5) * h + mn
    xr = pts[:, :3] + 2 * (xf - pts[:, :3])
    on_plane = (np.abs(((xr - mn) / h) % 1.0 - 0.5) < 1e-4).any(1)
    keep = same & ~on_plane
    assert keep.mean() > 0.95
    for rel in (0, -1):
        a, b = s.grid(rel).ravel(), o.grid(rel).ravel()
        np.testing.assert_allclose(a[keep], b[keep], rtol=1e-5, atol=1e-6)
    s.close()


def test_state_roundtrip_and_reset(gpu):
    s, o, v, f, h, mn, dt = _static_pair()
    s.add_listener(20, 20, 20)
    acc = sine_acc(80, len(f), 1500.0, dt)
    s.step(acc[:40])
    blob = s.save_state()
    t = s.t
    s.step(acc[40:])
    a = s.listeners()[40:, 0].copy()
    s.restore_state(blob)
    assert s.t == t
    s.rewind_listeners()
    s.step(acc[40:])
    assert np.array_equal(s.listeners()[:, 0], a)
    s.reset_fields()
    assert not np.any(s.grid(0)) and not np.any(s.dump("dirichlet"))
    s.close()


def test_bad_inputs_rejected(gpu):
    from pppm_b200 import PPPMError

    v, f, h, mn, dt = sphere_small()
    with pytest.raises(PPPMError):
        Solver(4, h, dt, mn)
    s = Solver(24, h, dt, mn)
    with pytest.raises(PPPMError):
        s.set_mesh(v, np.full_like(f, len(v)))  # index out of range
    with pytest.raises(PPPMError):
        s.set_mesh(v * 10, f)  # mesh leaves the grid interior
    s.close()
    s = Solver(24, h, dt, mn)
    s.set_mesh(v, f)
    with pytest.raises(PPPMError):
        s.step(None, nsteps=1)  # accelerations required once a mesh is set
    s.close()
