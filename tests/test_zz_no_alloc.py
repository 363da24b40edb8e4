"""pppm_pair_weights_static (single-pair weights on the library's static scratch, no device
allocation) against pppm_pair_weights (the same kernel on cudaMalloc'd scratch).  Collected
last so it also runs after every other GPU test has used the device."""
import numpy as np
import pytest

import pppm_b200
from pppm_b200 import PPPMError, pair_weights, pair_weights_static, scenes

pytestmark = pytest.mark.gpu

TOL = 1e-5  # of each layer's max-abs tap, as for the pair weights against the reference


def _cases():
    v, f = scenes.icosphere(2)
    v = (v * 0.1).astype(np.float32)
    h = np.float32(0.1 / 12)
    dt = np.float32(0.5 * h / (np.sqrt(3) * 340.3))
    t0 = f[0]
    share = [k for k in range(1, len(f)) if len(set(f[k]) & set(t0)) == 2][0]
    corner = [k for k in range(1, len(f)) if len(set(f[k]) & set(t0)) == 1][0]
    far = int(np.argmax(np.linalg.norm(v[f].mean(1) - v[t0].mean(0), axis=1)))
    cases = [dict(face=f[k]) for k in (0, share, corner, far)]
    cases.append(dict(point=v[t0].mean(0) + np.float32(1.3) * h))
    return dt, h, v, t0, cases


def _diff(a, b):
    worst = 0.0
    for half in (slice(0, 16), slice(16, 32)):
        sc = max(float(np.abs(b[half]).max()), 1e-30)
        worst = max(worst, float(np.abs(a[half] - b[half]).max()) / sc)
    return worst


def test_static_scratch_matches_allocating_entry_point(gpu):
    dt, h, v, src, cases = _cases()
    for case in cases:
        want = pair_weights(dt, h, v, src, **case)
        first = pair_weights_static(dt, h, v, src, **case)
        second = pair_weights_static(dt, h, v, src, **case)
        assert np.all(np.isfinite(want))
        assert _diff(first, want) < TOL
        assert _diff(second, want) < TOL


def test_static_scratch_rejects_too_many_vertices(gpu):
    dt, h, v, src, cases = _cases()
    big = np.zeros((pppm_b200.STATIC_MAX_VERTS + 1, 3), np.float32)
    big[: len(v)] = v
    with pytest.raises(PPPMError) as e:
        pair_weights_static(dt, h, big, src, **cases[0])
    assert e.value.status == pppm_b200.ERR_CAPACITY
    assert "static scratch limit" in str(e.value)
