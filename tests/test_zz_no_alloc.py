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


def test_static_scratch_beside_queued_steps_allocates_nothing(gpu):
    """The use the entry point exists for: a thread computes pair weights on its own non-blocking
    stream while a handle on the same device has steps queued.  After one warm-up call (which
    looks up the scratch address), calls change no device allocation, and the queued steps are
    not disturbed."""
    import torch

    from pppm_b200 import Solver

    dt, h, v, src, cases = _cases()
    want = [pair_weights(dt, h, v, src, **case) for case in cases]
    sv, sf = scenes.icosphere(2)
    sv = (sv * 0.1).astype(np.float32)
    res = 24
    gh, mn = scenes.grid_for_bbox(sv.min(0), sv.max(0), res, 2.0)
    gdt = np.float32(0.5 * gh / (np.sqrt(3) * 340.3))
    s = Solver(res, gh, gdt, mn)
    s.set_mesh(sv, sf)
    s.add_listener(20, 20, 20)
    acc = torch.ones((400, len(sf)), dtype=torch.float32, device="cuda")
    s.step(acc[:200])  # records the step graph (graph instantiation may allocate)
    torch.cuda.synchronize()
    s.rewind_listeners()  # the next 200 samples reuse the rows: no series growth below
    side = torch.cuda.Stream()
    pair_weights_static(dt, h, v, src, stream=side.cuda_stream, **cases[0])  # warm-up: address look-up
    free0 = torch.cuda.mem_get_info()[0]
    s.step(acc[200:])  # queued on the handle's stream; returns before the steps have run
    for _ in range(2):
        for case, w in zip(cases, want):
            got = pair_weights_static(dt, h, v, src, stream=side.cuda_stream, **case)
            assert _diff(got, w) < TOL
    free1 = torch.cuda.mem_get_info()[0]
    series = s.listeners()[:, 0]
    s.close()
    assert free1 == free0
    assert len(series) == 200 and np.all(np.isfinite(series))


def test_failed_call_restores_the_current_device(gpu):
    """A call for a device this process cannot use fails with a CUDA status and leaves the calling
    thread's current device as it was."""
    import torch

    dt, h, v, src, cases = _cases()
    before = torch.cuda.current_device()
    bad = torch.cuda.device_count()  # one past the last device
    with pytest.raises(PPPMError) as e:
        pair_weights_static(dt, h, v, src, device=bad, **cases[0])
    assert e.value.status in (pppm_b200.ERR_CUDA, pppm_b200.ERR_ARG)
    assert torch.cuda.current_device() == before
    got = pair_weights_static(dt, h, v, src, device=before, **cases[0])
    assert _diff(got, pair_weights(dt, h, v, src, **cases[0])) < TOL
