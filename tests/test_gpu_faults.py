"""Failure detection with host-made faults (no device fault is provoked): a NaN acceleration
reaches the step status word and is reported as PPPM_ERR_NAN by the next step call and by
pppm_sync, the fields can be reset and stepping goes on; a mesh whose face-pair list exceeds
the face cache's 1024 neighbours per face (the reference's PARTICLE_CACHE_SIZE,
pppm_cache.h:79) is refused with PPPM_ERR_CAPACITY and leaves the handle usable.  The reference
aborts the demo on a NaN listener sample (experiments/demo/main.cu:161-168)."""
import numpy as np
import pytest

import pppm_b200
from helpers import sine_acc, sphere_small
from pppm_b200 import PPPMError, Solver

pytestmark = pytest.mark.gpu


def _solver():
    v, f, h, mn, dt = sphere_small()
    s = Solver(24, h, dt, mn)
    s.set_mesh(v, f)
    s.add_listener(20, 20, 20)
    return s, f, dt


@pytest.mark.parametrize("on_device", [False, True])
def test_nan_acceleration_is_reported(gpu, on_device):
    import torch

    s, f, dt = _solver()
    acc = sine_acc(40, len(f), 1500.0, dt)
    acc[7, 5] = np.nan
    a = torch.from_numpy(acc).cuda() if on_device else acc
    s.step(a)  # queued; the flag is raised on the device
    with pytest.raises(PPPMError) as e:
        s.sync()
    assert e.value.status == pppm_b200.ERR_NAN
    with pytest.raises(PPPMError) as e:
        s.step(sine_acc(8, len(f), 1500.0, dt))
    assert e.value.status == pppm_b200.ERR_NAN
    s.reset_fields()
    s.rewind_listeners()
    s.step(sine_acc(40, len(f), 1500.0, dt))
    s.sync()
    assert np.all(np.isfinite(s.listeners()))
    s.close()


def test_finite_run_reports_nothing(gpu):
    s, f, dt = _solver()
    for _ in range(3):
        s.step(sine_acc(30, len(f), 1500.0, dt))
    s.sync()
    s.close()


def test_face_cache_overflow_is_refused(gpu):
    rng = np.random.default_rng(5)
    res, h = 16, np.float32(0.01)
    n = 1100  # triangles whose centres share one 4^3 block: each centre sees them all
    c = rng.uniform(0.075, 0.085, (n, 3))
    e1 = rng.normal(size=(n, 3)) * 1e-3
    e2 = rng.normal(size=(n, 3)) * 1e-3
    verts = np.concatenate([c, c + e1, c + e2]).astype(np.float32)
    tris = np.stack([np.arange(n), np.arange(n) + n, np.arange(n) + 2 * n], 1).astype(np.int32)
    dt = np.float32(0.5 * h / (np.sqrt(3) * 340.3))
    s = Solver(res, h, dt, (0.0, 0.0, 0.0))
    with pytest.raises(PPPMError) as e:
        s.set_mesh(verts, tris)
    assert e.value.status == pppm_b200.ERR_CAPACITY
    # the handle is still usable with a mesh inside the limits
    s.set_mesh(verts[[0, n, 2 * n]], np.array([[0, 1, 2]], np.int32))
    s.add_listener(3, 3, 3)
    s.step(np.ones((10, 1), np.float32))
    s.sync()
    assert np.all(np.isfinite(s.listeners()))
    s.close()
