"""PPPM_WEIGHTS_FP64 on the B200: an FP32 run whose singular face integrals (face pairs sharing a
vertex, an edge or the whole triangle: the Sauter-Schwab rules of integrand.h:51-173) are
evaluated in FP64 before the fp16 packing, against the FP64 scheme of this library (unquantised
FP64 weights everywhere), beside the default mode that evaluates them with the reference's FP32
arithmetic.

  * regular pairs (no shared vertex) are computed the same way in both modes: bit-identical
    records;
  * singular pairs: each mode's taps against the FP64 scheme's, relative to the record's max-abs
    tap (both layers: the double layer of an identical pair is analytically zero, ~1e-19 in
    FP64, so a per-layer scale would compare rounding noise); the FP64 mode within the fp16
    packing bound (2^-11 of the record scale) and closer than the FP32 mode on average;
  * the listener series of each mode against the FP64 run (300 steps).

Measured figures go to $PPPM_METRICS_DIR/fp64_weights_metrics.json when that variable is set.
"""
import json
import os

import numpy as np
import pytest

from helpers import records_to_taps, rel_l2, sine_acc, sphere_small
from pppm_b200 import Solver

pytestmark = pytest.mark.gpu


def _run(weights=None, precision="fp32", steps=300):
    v, f, h, mn, dt = sphere_small()
    kw = {"precision": precision}
    if weights:
        kw["weights"] = weights
    s = Solver(24, h, dt, mn, **kw)
    s.set_mesh(v, f)
    s.add_listener(20, 20, 20)
    pairs = s.dump("face_pairs").reshape(-1, 2)
    rec = s.dump("face_cache")
    s.step(sine_acc(steps, len(f), 1500.0, dt))
    series = s.series()[:, 0].astype(np.float64)
    s.close()
    return f, pairs, rec, series


def _row_err(taps, ref):
    """per record: max |taps - ref| / max |ref| over both layers"""
    return np.abs(taps - ref).max(1) / np.maximum(np.abs(ref).max(1), 1e-30)


def test_fp64_singular_weights(gpu):
    f, p64, r64, s64 = _run(precision="fp64")
    f, p32, r32, s32 = _run("ref32")
    _, pw, rw, sw = _run("fp64")
    assert np.array_equal(p32, p64) and np.array_equal(pw, p64)
    ref = np.concatenate([r64[:, :, 0], r64[:, :, 1]], 1)  # FP64 records: taps x (single, double)
    t32, tw = records_to_taps(r32).astype(np.float64), records_to_taps(rw).astype(np.float64)
    shared = np.array([len(set(f[a]) & set(f[b])) for a, b in p64])
    sing = shared > 0
    regular_equal = bool(np.array_equal(r32.view(np.uint8).reshape(-1, 72)[~sing],
                                        rw.view(np.uint8).reshape(-1, 72)[~sing]))
    e32, ew = _row_err(t32[sing], ref[sing]), _row_err(tw[sing], ref[sing])
    m = {"singular_pairs": int(sing.sum()), "pairs": int(len(p64)), "regular_records_bit_identical": regular_equal,
         "singular_max_err_ref32": float(e32.max()), "singular_max_err_fp64": float(ew.max()),
         "singular_mean_err_ref32": float(e32.mean()), "singular_mean_err_fp64": float(ew.mean()),
         "listener_rel_l2_vs_fp64_scheme_ref32": rel_l2(s32, s64), "listener_rel_l2_vs_fp64_scheme_fp64": rel_l2(sw, s64)}
    d = os.environ.get("PPPM_METRICS_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "fp64_weights_metrics.json"), "w") as fo:
            json.dump(m, fo, indent=1)
    assert sing.sum() > 0
    assert regular_equal
    assert ew.max() < 2.0 ** -11  # fp16 packing of the FP64 integrals
    assert ew.mean() < e32.mean()
    assert np.all(np.isfinite(sw))
    assert rel_l2(sw, s64) < rel_l2(s32, s64)
