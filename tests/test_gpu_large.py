"""The large moving scene on the B200: res 128 (2.1 M cells), two perturbed icospheres of
20480 triangles each on independent seeded rigid trajectories, band-limited noise
accelerations on both, 1 kHz motion frames (pppm_b200.scenes.LargeScene).

  * against the reference solver compiled from source (oracle/_ref, on the same GPU): per-cell
    3^3 lists bit-exact after the last motion frame, and the listener series over the first
    motion frames (own weight tables on each side; the reference sums its corrections with
    float atomics, so its own repeats differ in the last bits and the scheme amplifies that);
  * the whole 20000-step run (about 245 motion frames) in FP32 against the same run in the FP64
    scheme of this library, the error yardstick every FP32 result is quoted against: relative
    L2 of the listener series <= 2e-2 (the FP32 scheme stores its weights as fp16 rows), and
    every sample finite.

Measured figures are written to $PPPM_METRICS_DIR/large_metrics.json when that variable is set.
"""
import json
import os

import numpy as np
import pytest

from helpers import per_cell_sets, rel_l2
from pppm_b200 import Solver, scenes

pytestmark = pytest.mark.gpu
METRICS = {}


@pytest.fixture(scope="module", autouse=True)
def write_metrics():
    yield
    d = os.environ.get("PPPM_METRICS_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "large_metrics.json"), "w") as f:
            json.dump(METRICS, f, indent=1, default=float)


@pytest.fixture(scope="module")
def scene():
    return scenes.LargeScene()


def _run(sc, ranges, precision="fp32", device_acc=True):
    import torch

    s = Solver(sc.res, sc.h, sc.dt, sc.min_pos, precision=precision)
    s.set_mesh(sc.frame_verts(0), sc.tris)
    s.add_listener(*sc.listener)
    for f, (a, b) in enumerate(ranges):
        if f:
            s.update_mesh(sc.frame_verts(f))
        acc = sc.acc(a, b - a)
        s.step(torch.from_numpy(acc).cuda() if device_acc else acc)
    return s


def test_large_scene_vs_reference(gpu, scene):
    from oracle import oracle as O

    if not O.reference_available():
        pytest.skip("reference solver not built (make -C oracle ref)")
    sc = scene
    nframes = 3
    ranges = scenes.frame_ranges(sc, nframes - 1)
    s = _run(sc, ranges)
    got = s.listeners()[:, 0]
    n3 = s.dump("n3_cells").reshape(-1, 4)
    ours_lists = per_cell_sets(n3, s.dump("n3_tris"))
    counts = [int(x) for x in s.dump("counts")]
    s.close()

    r = O.Reference(sc.res, sc.h, sc.dt, sc.min_pos)
    try:
        r.set_mesh(sc.frame_verts(0), sc.tris)  # set_mesh and update_mesh check the reference's capacities
        ref = []
        for f, (a, b) in enumerate(ranges):
            if f:
                r.update_mesh(sc.frame_verts(f))
            ref.append(r.run(sc.acc(a, b - a), [sc.listener])[:, 0])
        ref = np.concatenate(ref)
        L = r.lists()
    finally:
        r.close()
    assert ours_lists == per_cell_sets(L["n3_cells"], L["n3_tris"])
    err = rel_l2(got, ref)
    METRICS["vs_reference"] = {"steps": int(len(got)), "frames": nframes, "rel_l2": err,
                               "rel_l2_first50": rel_l2(got[:50], ref[:50]), "n3_cells": counts[0],
                               "pairs_3x3x3": counts[1], "face_pairs": counts[4]}
    assert np.all(np.isfinite(got))
    assert err < 1e-3


def test_large_scene_full_run_fp32_vs_fp64(gpu, scene):
    sc = scene
    nframes = sc.frame_of_step(sc.steps - 1) + 1
    ranges = scenes.frame_ranges(sc, nframes - 1)
    ranges[-1] = (ranges[-1][0], sc.steps)
    out = {}
    for prec in ("fp32", "fp64"):
        s = _run(sc, ranges, precision=prec)
        out[prec] = s.listeners()[:, 0]
        s.close()
    assert len(out["fp32"]) == sc.steps
    assert np.all(np.isfinite(out["fp32"]))
    err = rel_l2(out["fp32"], out["fp64"])
    METRICS["fp32_vs_fp64"] = {"steps": sc.steps, "frames": nframes, "rel_l2": err,
                               "rms_fp64": float(np.sqrt(np.mean(np.asarray(out["fp64"], np.float64) ** 2)))}
    assert err < 2e-2
