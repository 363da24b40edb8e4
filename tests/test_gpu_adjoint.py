"""Adjoint of the step (pppm_adjoint) and its torch.autograd bridge.

The listener samples of a run from the zero state are a linear function of the accelerations,
series = A acc, so the adjoint must satisfy <g, A x> = <A^T g, x> for any x and g, and equal
the Jacobian built column by column from unit impulses; both are checked in FP64 to ~1e-10.
The gradient of a least-squares loss is checked against central finite differences of the
forward along random directions (FP64: 1e-9; FP32: 1e-3) and the FP32 gradient against the FP64
one.  Inputs and directions are dyadic (multiples of 2^-10), so x +- eps v is exact in float32
and the difference quotient of the quadratic loss is centred on x itself.

When PPPM_METRICS_DIR is set the measured errors go to adjoint_metrics.json there.
"""
import json
import os

import numpy as np
import pytest

from helpers import dyadic, sphere_small
from pppm_b200 import PPPMError, Solver

pytestmark = pytest.mark.gpu

METRICS = {}


def _record(key, value):
    METRICS[key] = value
    d = os.environ.get("PPPM_METRICS_DIR")
    if d:
        with open(os.path.join(d, "adjoint_metrics.json"), "w") as f:
            json.dump(METRICS, f, indent=1)


def _solver(precision="fp64", res=20, sub=1, shell_listener=True, pml_width=0):
    v, f, h, mn, dt = sphere_small(res, sub)
    s = Solver(res, h, dt, mn, precision=precision, pml_width=pml_width)
    s.set_mesh(v, f)
    s.add_listener(res - 4, res - 4, res - 4)  # far field
    c = s.dump("n3_cells").reshape(-1, 4)[0]
    s.add_listener(int(c[0]), int(c[1]), int(c[2]))  # a corrected cell
    if shell_listener:
        s.add_listener(1, res // 2, res // 3)  # boundary layer (inside the PML when there is one)
    if pml_width:
        s.add_listener(res - 2 - pml_width // 2, res // 2 + 1, res // 2)  # inside the PML, upper side
    return s


def _forward(s, x):
    """series of len(x) steps from the zero state"""
    s.reset_fields()
    s.rewind_listeners()
    s.step(x)
    return s.series(0, len(x)).astype(np.float64)


def test_dot_product_fp64(gpu):
    s = _solver("fp64")
    n = 90  # long enough for waves to reach the boundary layer and come back
    rng = np.random.default_rng(1)
    x = rng.standard_normal((n, s.nt)).astype(np.float32)
    g = rng.standard_normal((n, s.n_listeners))
    y = _forward(s, x)
    gx = s.adjoint(g)
    lhs, rhs = float(np.sum(g * y)), float(np.sum(gx * x.astype(np.float64)))
    scale = float(np.sum(np.abs(g * y)))
    _record("dot_product_fp64_rel", abs(lhs - rhs) / scale)
    assert abs(lhs - rhs) <= 1e-10 * scale, (lhs, rhs)
    s.close()


def test_jacobian_fp64(gpu):
    """Every column of the Jacobian from a unit impulse, against J^T g from the adjoint."""
    s = _solver("fp64", res=16, sub=0)
    n, nt = 14, s.nt
    J = np.zeros((n, s.n_listeners, n, nt))
    e = np.zeros((n, nt), np.float32)
    for k in range(n):
        for j in range(nt):
            e[k, j] = 1.0
            J[:, :, k, j] = _forward(s, e)
            e[k, j] = 0.0
    rng = np.random.default_rng(2)
    worst = 0.0
    for trial in range(3):
        g = rng.standard_normal((n, s.n_listeners))
        want = np.einsum("sl,slkj->kj", g, J)
        got = s.adjoint(g)
        err = np.abs(got - want).max() / np.abs(want).max()
        worst = max(worst, float(err))
        if err > 1e-10:
            d = os.environ.get("PPPM_METRICS_DIR")
            if d:
                np.savez(os.path.join(d, "adjoint_jacobian_fail.npz"), J=J, g=g, got=got, want=want)
    # each listener and step on its own: the rows of J
    for sl in [(n - 1, 0), (n - 1, 1), (n - 5, 2), (0, 1)]:
        g = np.zeros((n, s.n_listeners))
        g[sl] = 1.0
        got = s.adjoint(g)
        want = J[sl[0], sl[1]]
        err = np.abs(got - want).max() / max(np.abs(want).max(), 1e-300)
        worst = max(worst, float(err))
    _record("jacobian_fp64_max_rel", worst)
    assert worst <= 1e-10
    s.close()


def test_chunks_continue_the_sweep(gpu):
    s = _solver("fp64")
    n = 70
    g = np.random.default_rng(3).standard_normal((n, s.n_listeners))
    whole = s.adjoint(g)
    last = s.adjoint(g[50:], fresh=True)
    mid = s.adjoint(g[20:50], fresh=False)
    first = s.adjoint(g[:20], fresh=False)
    assert np.array_equal(np.concatenate([first, mid, last]), whole)
    s.close()


@pytest.mark.parametrize("pml", [0, 4])
def test_recorded_chunks_match_direct_launches(gpu, pml):
    """A long sweep replays a recorded chunk of 32 reverse steps (the kernels read their time
    from device memory) and launches the rest directly; the same sweep in calls of 50 steps, which
    launch every kernel directly, gives bit-identical gradients."""
    s = _solver("fp32", res=20, sub=1, pml_width=pml)
    n = 300
    g = np.random.default_rng(8).standard_normal((n, s.n_listeners))
    whole = s.adjoint(g)
    parts = []
    for k, e in enumerate(range(n, 0, -50)):
        parts.append(s.adjoint(g[e - 50:e], fresh=(k == 0)))
    assert np.array_equal(np.concatenate(parts[::-1]), whole)
    assert np.all(np.isfinite(whole)) and np.abs(whole).max() > 0
    s.close()


def _fd_check(s, acc, target, grad, rng, ndir):
    """worst relative gap between <grad, v> and central differences of the loss along v"""

    def loss(x):
        return float(np.sum((_forward(s, x) - target) ** 2))

    worst = 0.0
    for _ in range(ndir):
        v = dyadic(rng, acc.shape)
        eps = 0.125
        xp, xm = acc + np.float32(eps) * v, acc - np.float32(eps) * v  # exact in float32 (dyadic inputs)
        assert np.array_equal((xp.astype(np.float64) + xm) / 2, acc)
        fd = (loss(xp) - loss(xm)) / (2 * eps)
        an = float(np.sum(grad * v.astype(np.float64)))
        worst = max(worst, abs(fd - an) / max(abs(fd), 1e-300))
    return worst


def test_gradient_vs_finite_differences(gpu):
    """Loss ||s - s_target||^2: each precision's adjoint gradient against central differences of
    its own forward along random directions; the FP32 gradient against the FP64 one (the FP32
    scheme stores its weights as fp16 + scale, so the two schemes differ at that level)."""
    n = 120
    s32, s64 = _solver("fp32", res=24, sub=2), _solver("fp64", res=24, sub=2)
    rng = np.random.default_rng(4)
    acc = dyadic(rng, (n, s32.nt))
    # a target on the signal's scale, so the difference quotient does not cancel
    target = rng.standard_normal((n, s32.n_listeners)) * _forward(s64, acc).std()
    grad32 = s32.adjoint(2 * (_forward(s32, acc) - target))
    grad64 = s64.adjoint(2 * (_forward(s64, acc) - target))
    fd64 = _fd_check(s64, acc, target, grad64, rng, 16)
    fd32 = _fd_check(s32, acc, target, grad32, rng, 16)
    rel = float(np.linalg.norm(grad32 - grad64) / np.linalg.norm(grad64))
    _record("fp64_vs_fd_max_rel", fd64)
    _record("fp32_vs_fd_max_rel", fd32)
    _record("fp32_vs_fp64_adjoint_rel_l2", rel)
    assert fd64 <= 1e-9
    assert fd32 <= 1e-3
    assert rel <= 1e-2
    s32.close()
    s64.close()


def test_autograd_chunks(gpu):
    import torch

    from pppm_b200.autograd import listener_signal

    s = _solver("fp32", res=20, sub=1)
    rng = np.random.default_rng(5)
    a1 = torch.tensor(rng.standard_normal((40, s.nt)), dtype=torch.float32, device="cuda", requires_grad=True)
    a2 = torch.tensor(rng.standard_normal((35, s.nt)), dtype=torch.float32, device="cuda", requires_grad=True)
    w = torch.tensor(rng.standard_normal((35, s.n_listeners)), dtype=torch.float32, device="cuda")
    sig1, tok = listener_signal(s, a1)
    sig2, tok = listener_signal(s, a2, tok)
    loss = (sig1 ** 2).sum() + (sig2 * w).sum()
    loss.backward()
    g = np.concatenate([2 * sig1.detach().cpu().numpy(), w.cpu().numpy()])
    want = s.adjoint(g)
    got = np.concatenate([a1.grad.cpu().numpy(), a2.grad.cpu().numpy()])
    assert np.allclose(got, want, rtol=1e-5, atol=1e-6 * np.abs(want).max())
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_pml_dot_product(gpu, precision):
    """The split-field PML (fdtd.cu:179-232) transposed: <g, A x> = <A^T g, x> over a run long
    enough for the waves to enter the layer and for its auxiliary fields to feed back, with
    listeners in the field, at a corrected cell, on the boundary layer and inside the PML."""
    s = _solver(precision, res=20, pml_width=4)
    n = 110
    rng = np.random.default_rng(6)
    x = rng.standard_normal((n, s.nt)).astype(np.float32)
    g = rng.standard_normal((n, s.n_listeners))
    y = _forward(s, x)
    gx = s.adjoint(g)
    lhs, rhs = float(np.sum(g * y)), float(np.sum(gx * x.astype(np.float64)))
    scale = float(np.sum(np.abs(g * y)))
    _record("pml_dot_product_%s_rel" % precision, abs(lhs - rhs) / scale)
    # FP64: the exact transpose; FP32: the forward rounds in float, the adjoint of the exact map
    assert abs(lhs - rhs) <= (1e-10 if precision == "fp64" else 1e-4) * scale, (lhs, rhs)
    s.close()


def test_pml_gradient_vs_finite_differences(gpu):
    n = 100
    s32, s64 = _solver("fp32", res=22, sub=1, pml_width=4), _solver("fp64", res=22, sub=1, pml_width=4)
    rng = np.random.default_rng(7)
    acc = dyadic(rng, (n, s32.nt))
    target = rng.standard_normal((n, s32.n_listeners)) * _forward(s64, acc).std()
    grad32 = s32.adjoint(2 * (_forward(s32, acc) - target))
    grad64 = s64.adjoint(2 * (_forward(s64, acc) - target))
    fd64 = _fd_check(s64, acc, target, grad64, rng, 8)
    fd32 = _fd_check(s32, acc, target, grad32, rng, 8)
    _record("pml_fp64_vs_fd_max_rel", fd64)
    _record("pml_fp32_vs_fd_max_rel", fd32)
    assert fd64 <= 1e-9
    assert fd32 <= 1e-3
    s32.close()
    s64.close()


def test_adjoint_rejects(gpu):
    v, f, h, mn, dt = sphere_small(24, 1)
    s = Solver(24, h, dt, mn)
    s.set_mesh(v, f)
    s.add_listener(0, 12, 12)  # outer ghost layer: no sample is ever recorded there
    with pytest.raises(PPPMError):
        s.adjoint(np.zeros((4, 1)))
    s.close()
