"""The algebra of the two-step passes of the recorded step graphs, restated in numpy (float64) on
random data, and the autotuner's option-set numbering.

Face pairs (step.cu: face_conv2 + face_fix): a centre's convolution at time t is
    sum_j sum_k ( -s_jk N_j[t-k] + d_jk D_j[t-k] ),  k = 0..15, with D_j[t] (unknown) left out.
At time t+1 every term is known before step t except d_j1 D_j[t]; the pass computes the rest from
the time-t windows shifted by one tap (tap -1 = N[t+1]) and adds sum_j d_j1 D_j[t] afterwards.

Grid-cache records (step.cu: near_terms2 + near_terms_complete): BEM-near terms pair record tap m
with history tap m, FDTD-near terms with history tap m-1; at time t+1 the only unknown product is
the one with D[t+1] (record tap 0, resp. 1), added from one factor per record afterwards.
"""
import numpy as np

from pppm_b200 import Solver

TAPS = 16


def _history(rng, n, t):
    """N[tau], D[tau] for tau = t-31 .. t+1 (dict-like arrays indexed by tau - (t - 31))."""
    return rng.standard_normal((n, 33)), rng.standard_normal((n, 33))


def _at(h, t, tau):
    return h[..., tau - (t - 31)]


def test_face_pair_two_step_identity():
    rng = np.random.default_rng(3)
    npair, t = 40, 100
    s = rng.standard_normal((npair, TAPS))
    d = rng.standard_normal((npair, TAPS))
    N, D = _history(rng, npair, t)

    def conv(time):  # one pass, D[time] left out (it is the step's unknown)
        acc = 0.0
        for k in range(TAPS):
            dk = 0.0 if k == 0 else _at(D, t, time - k)
            acc += np.sum(-s[:, k] * _at(N, t, time - k) + d[:, k] * dk)
        return acc

    # the two-step pass: time-t windows (taps t .. t-15), shifted by one for time t+1
    hn = np.stack([_at(N, t, t - k) for k in range(TAPS)], 1)
    hd = np.stack([_at(D, t, t - k) for k in range(TAPS)], 1)
    hd[:, 0] = 0.0  # D[t] unknown at conv time
    c0 = np.sum(-s * hn + d * hd)
    sn = np.concatenate([_at(N, t, t + 1)[:, None], hn[:, :-1]], 1)  # tap 0 of t+1 is N[t+1]
    sd = np.concatenate([np.zeros((npair, 2)), hd[:, 1:-1]], 1)  # D[t+1] and D[t] left out
    partial = np.sum(-s * sn + d * sd)
    fix = np.sum(d[:, 1] * _at(D, t, t))  # D[t] known after finish(t)
    assert abs(c0 - conv(t)) < 1e-12 * max(1.0, abs(c0))
    assert abs(partial + fix - conv(t + 1)) < 1e-12 * max(1.0, abs(partial))


def test_near_terms_two_step_identity():
    rng = np.random.default_rng(4)
    t = 50
    w_s = rng.standard_normal((54, TAPS))
    w_d = rng.standard_normal((54, TAPS))
    N, D = _history(rng, 1, t)
    N, D = N[0], D[0]

    def term(r, time):  # one pass: BEM-near (r >= 27) taps m; FDTD-near (r < 27) record tap m, history m-1
        acc = 0.0
        for m in range(TAPS):
            k = m if r >= 27 else m - 1
            if k < 0:
                continue
            acc += -w_s[r, m] * _at(N, t, time - k) + w_d[r, m] * _at(D, t, time - k)
        return acc

    # partial terms of time t+1 from the time-t window, D[t+1] left out, then completed
    for r in range(54):
        partial = 0.0
        for m in range(TAPS):
            k = m if r >= 27 else m - 1
            if k < 0:
                continue
            tau = t + 1 - k
            dval = 0.0 if tau == t + 1 else _at(D, t, tau)
            partial += -w_s[r, m] * _at(N, t, tau) + w_d[r, m] * dval
        factor = w_d[r, 0] if r >= 27 else w_d[r, 1]
        full = partial + factor * _at(D, t, t + 1)
        assert abs(full - term(r, t + 1)) < 1e-12 * max(1.0, abs(full))


def test_autotune_config_numbering():
    # config j of phase 2: conv_pairs = j / 6, threads = {64, 128, 256}[(j / 2) % 3], terms = j % 2
    for j, (pairs, threads, terms) in enumerate(Solver.TUNE_CONFIGS):
        assert (pairs, threads, terms) == (j // 6, (64, 128, 256)[(j // 2) % 3], j % 2)
    for i, (pairs, threads) in enumerate(Solver.TUNE_CANDIDATES):
        assert (pairs, threads) == (i // 3, (64, 128, 256)[i % 3])
