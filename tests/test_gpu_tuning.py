"""Launch options of the recorded step graphs and the face-stage autotuner, on the B200.

The two-step face-pair convolution (conv2 + fix: one pass over the pairs' weights for two
consecutive steps) sums the same products as one pass per step, with the term of D[t] added after
the rest instead of among it.  Tolerances: FP64 series of the two variants within 1e-12 relative
L2 over 300 steps (the algebra is the same); FP32 within 1e-6 over the first 50 steps and 1e-4
over 300 (reassociation only: the scheme amplifies rounding differences step after step, and
summing the same pairs in reverse order already moves a 300-step FP32 series by ~3e-5); both
within the oracle bounds of the parity tests (1e-5 over the first 50 steps with shared tables)."""
import numpy as np
import pytest

from helpers import edge_sphere, moving_small_verts, rel_l2, sine_acc, sphere_small
from oracle.oracle import Oracle
from pppm_b200 import Solver

pytestmark = pytest.mark.gpu


def _series(precision, pairs, threads=256, steps=300, chunk=None, moving=False, terms=None, split=1,
            graph_chunk=None, vec4=None):
    v0, f, h, mn, dt = sphere_small()
    res = 24
    s = Solver(res, h, dt, mn, precision=precision)
    s.set_option("split_stencil", split)
    if graph_chunk is not None:
        s.set_option("graph_chunk", graph_chunk)
    if vec4 is not None:
        s.set_option("stencil_vec4", vec4)
    s.set_option("conv_pairs", pairs)
    s.set_option("terms_pairs", (1 if pairs else 0) if terms is None else terms)
    s.set_option("face_threads", threads)
    s.set_mesh(moving_small_verts(v0, 0, dt) if moving else v0, f)
    s.add_listener(20, 20, 20)
    acc = sine_acc(steps, len(f), 1500.0, dt)
    chunk = chunk or steps
    for s0 in range(0, steps, chunk):
        if moving and s0:
            s.update_mesh(moving_small_verts(v0, s0, dt))
        s.step(acc[s0: s0 + chunk])
    out = s.listeners()[:, 0].astype(np.float64)
    s.close()
    return out


def test_pairs_match_single_pass_fp64(gpu):
    a = _series("fp64", 0)
    b = _series("fp64", 1)
    assert np.all(np.isfinite(b))
    assert rel_l2(b, a) < 1e-12


@pytest.mark.parametrize("conv,terms", [(1, 0), (0, 1)])
def test_pairing_each_stage_fp64(gpu, conv, terms):
    # the convolution and the near-field terms pair their steps independently
    a = _series("fp64", 0, terms=0)
    b = _series("fp64", conv, terms=terms)
    assert rel_l2(b, a) < 1e-12


def test_pairs_match_single_pass_fp32(gpu):
    a = _series("fp32", 0)
    b = _series("fp32", 1)
    assert np.all(np.isfinite(b))
    assert rel_l2(b[:50], a[:50]) < 1e-6
    assert rel_l2(b, a) < 1e-4


@pytest.mark.parametrize("chunk", [5, 7, 13])
def test_pairs_odd_calls_and_motion(gpu, chunk):
    # odd step counts end a call on a single pass; motion frames change the pair lists between
    # calls (the tap-1 factors are rebuilt with the weights)
    a = _series("fp64", 0, steps=120, chunk=chunk, moving=True)
    b = _series("fp64", 1, steps=120, chunk=chunk, moving=True)
    assert rel_l2(b, a) < 1e-12


@pytest.mark.parametrize("pairs,threads", [(1, 64), (1, 128), (0, 64)])
def test_face_threads(gpu, pairs, threads):
    a = _series("fp32", pairs)
    b = _series("fp32", pairs, threads=threads)
    assert np.array_equal(a, b)  # same arithmetic, other block shape


def test_autotune_keeps_results(gpu):
    v, f, h, mn, dt = sphere_small()
    res = 24
    s = Solver(res, h, dt, mn)
    s.set_mesh(v, f)
    s.add_listener(20, 20, 20)
    acc = sine_acc(200, len(f), 1500.0, dt)
    s.step(acc[:100])
    t_before = s.t
    before = [s.grid(r).copy() for r in (0, -1, -2)] + [s.dump("neumann"), s.dump("dirichlet"), s.listeners()]
    tune = s.autotune(reps=3)
    assert len(tune["us"]) == 6 and all(u > 0 for u in tune["us"].values())
    # phase 2 (whole recorded steps of every option set) decides
    assert tune["step_us"] is not None and len(tune["step_us"]) == 12
    assert all(u > 0 for u in tune["step_us"].values())
    chosen = (s.get_option("conv_pairs"), s.get_option("face_threads"), s.get_option("terms_pairs"))
    assert chosen == min(tune["step_us"], key=tune["step_us"].get)
    # fields, histories, time and recorded samples are as before
    after = [s.grid(r) for r in (0, -1, -2)] + [s.dump("neumann"), s.dump("dirichlet"), s.listeners()]
    assert s.t == t_before
    for x, y in zip(before, after):
        assert np.array_equal(x, y)
    s.step(acc[100:])
    got = s.listeners()[:, 0]
    s.close()
    o = Oracle(res, h, dt, mn)
    o.set_mesh(v, f)
    s2 = Solver(res, h, dt, mn)
    s2.set_mesh(v, f)
    o.import_grid_cache(s2.dump("grid_cache"))
    o.import_face_cache(s2.dump("face_pairs").reshape(-1, 2), s2.dump("face_cache"))
    s2.close()
    ref = o.step(acc, listeners=[(20, 20, 20)])[:, 0]
    o.close()
    assert rel_l2(got[:50], ref[:50]) < 1e-5
    assert rel_l2(got, ref) < 1e-3


def test_bad_options_rejected(gpu):
    v, f, h, mn, dt = sphere_small()
    s = Solver(24, h, dt, mn)
    from pppm_b200 import PPPMError

    with pytest.raises(PPPMError):
        s.set_option("face_threads", 96)
    with pytest.raises(PPPMError):
        s.set_option("conv_pairs", 2)
    with pytest.raises(PPPMError):
        s.set_option("terms_pairs", -1)
    for bad in (1, 7, -2, 8192):  # chunks hold whole pairs of steps
        with pytest.raises(PPPMError):
            s.set_option("graph_chunk", bad)
    for bad in (2, -2):
        with pytest.raises(PPPMError):
            s.set_option("stencil_vec4", bad)
    with pytest.raises(PPPMError):
        s.autotune()  # no mesh yet
    s.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_kernel_timing_leaves_the_run_unchanged(gpu, precision):
    """pppm_time_kernels between two step calls (each kernel kind of the next step launched back
    to back, then the state the next step reads rebuilt): the series and fields are bit-identical
    to the same run without it, and every kind gets a positive duration."""
    v0, f, h, mn, dt = sphere_small()
    acc = sine_acc(120, len(f), 1500.0, dt)
    out = []
    for timed in (False, True):
        s = Solver(24, h, dt, mn, precision=precision)
        s.set_mesh(v0, f)
        s.add_listener(20, 20, 20)
        s.step(acc[:60])
        if timed:
            t = s.time_kernels(5)
            for k in ("stencil", "conv", "conv2", "fix", "finish", "finish1", "finish2", "near", "face"):
                assert t.get(k, 0) > 0, (k, t)
        s.step(acc[60:])
        out.append((s.listeners(), s.grid(0), s.grid(-1), s.dump("dirichlet")))
        s.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("pairs", [0, 1])
@pytest.mark.parametrize("call", [300, 69, 37])
def test_graph_chunks_are_bit_identical(gpu, pairs, call):
    """A long call replayed as chunk graphs plus a remainder graph (chunks of 32 and of 6 steps)
    gives exactly the series of one graph per call, across motion frames and uneven call
    lengths (the pairs of steps and the call's last-step work are the same)."""
    a = _series("fp32", pairs, chunk=call, moving=True, graph_chunk=0)
    for g in (32, 6):
        b = _series("fp32", pairs, chunk=call, moving=True, graph_chunk=g)
        assert np.array_equal(a, b), (g, call)


@pytest.mark.parametrize("split", [0, 1])
def test_stencil_vec4_is_bit_identical(gpu, split):
    """The interior stencil four cells per thread (16-byte loads) against one cell per thread: the
    same arithmetic per cell, so the series are bit-identical, split or not, moving or not."""
    for moving in (False, True):
        a = _series("fp32", 1, steps=150, chunk=23, moving=moving, split=split, vec4=0)
        b = _series("fp32", 1, steps=150, chunk=23, moving=moving, split=split, vec4=1)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_split_stencil_is_bit_identical(gpu, precision):
    """The corrected-cell stencil on the critical branch plus the bulk beside it computes every cell
    with the same arithmetic as one stencil launch: series bit-identical, across motion frames and
    call lengths that leave single steps."""
    for moving in (False, True):
        a = _series(precision, 1, steps=150, chunk=23, moving=moving, split=0)
        b = _series(precision, 1, steps=150, chunk=23, moving=moving, split=1)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("split", [0, 1])
def test_measurement_mode_profiles_every_kernel(gpu, split):
    """Measurement mode (pppm_enable_timing) with the split face stage: groups of four steps replay
    the recorded graph's kernels serialised with events between them; every kind is counted once
    per launch and timed, and the run stays finite."""
    v0, f, h, mn, dt = sphere_small()
    s = Solver(24, h, dt, mn)
    s.set_option("split_stencil", split)
    s.set_option("conv_pairs", 1)
    s.set_option("terms_pairs", 1)
    s.set_mesh(v0, f)
    s.add_listener(20, 20, 20)
    s.enable_timing(True)
    s.step(sine_acc(42, len(f), 1500.0, dt))  # 10 groups of 4 steps, then 2 steps of the fused kernels
    prof = s.kernel_profile()
    s.enable_timing(False)
    assert np.all(np.isfinite(s.listeners()))
    s.close()
    n = {k: c for k, (us, c) in prof.items()}
    assert all(us > 0 for us, c in prof.values()), prof
    if split:
        assert n["stencil_bulk"] == 40 and n["stencil_corr"] == 40 and n["stencil"] == 2
    else:
        assert n["stencil"] == 42 and "stencil_bulk" not in n
    assert n["conv2"] == 20 and n["fix"] == 20 and n["near"] == 42 and n["face"] == 2
    assert n["finish1"] == 20 and n["finish2"] == 10 and n["finish"] == 10
    assert n["nwrite"] == 10 and n["empty"] == 10


def _edge_series(axis, cell, split, steps=150, chunk=23, profile=False):
    v, f, h, mn, dt = edge_sphere(axis, cell)
    s = Solver(24, h, dt, mn)
    s.set_option("split_stencil", split)
    s.set_option("conv_pairs", 1)
    s.set_option("terms_pairs", 1)
    s.set_mesh(v, f)
    s.add_listener(20, 12, 12)
    s.add_listener(1, 12, 12)
    acc = sine_acc(steps, len(f), 1500.0, dt)
    if profile:
        s.enable_timing(True)
    for s0 in range(0, steps, chunk):
        s.step(acc[s0: s0 + chunk])
    prof = s.kernel_profile() if profile else None
    out = s.listeners().astype(np.float64), s.grid(0).copy()
    s.close()
    return out, prof


@pytest.mark.parametrize("axis,cell,split", [(0, 3, False), (1, 20, False), (2, 3, False), (0, 4, True),
                                             (1, 19, True)])
def test_split_stencil_off_near_the_boundary(gpu, axis, cell, split):
    """A corrected cell two cells from the grid's face is the inward neighbour of a boundary-layer
    cell that is not corrected: that cell's 4x4 solve reads p^{t-1} there, which the split step's
    near stage overwrites with the next step's sums beside the bulk.  Such a mesh (a triangle in
    cell 3 or res-4 of an axis) runs the step unsplit, with the same results; one cell further in,
    the split stays."""
    (a, ga), prof = _edge_series(axis, cell, 1, steps=42, chunk=42, profile=True)
    n = {k: c for k, (us, c) in prof.items()}
    if split:
        assert n["stencil_bulk"] == 40 and n["stencil_corr"] == 40
    else:
        assert n["stencil"] == 42 and "stencil_bulk" not in n
    (b, gb), _ = _edge_series(axis, cell, 1)
    (c, gc), _ = _edge_series(axis, cell, 0)
    assert np.all(np.isfinite(b)) and np.abs(b).max() > 0
    assert np.array_equal(b, c) and np.array_equal(gb, gc)
