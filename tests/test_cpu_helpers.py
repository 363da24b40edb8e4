"""The vectorised list comparisons the whole-run GPU tests use (tests/helpers.py) against the
plain per-cell comparison, on the reference's own lists of the small sphere (golden fixture)."""
import numpy as np

from helpers import cell_list_codes, face_pair_codes, golden, per_cell_sets, window_counts


def test_list_codes_match_per_cell_sets():
    g = golden("sphere_small.npz")
    res, nt = int(g["res"]), len(g["tris"])
    codes = cell_list_codes(g["n3_cells"], g["n3_tris"], res, nt)
    sets = per_cell_sets(g["n3_cells"], g["n3_tris"])
    want = np.sort(np.array([((x * res + y) * res + z) * nt + t for (x, y, z), lst in sets.items() for t in lst]))
    assert np.array_equal(codes, want)
    # a permutation inside a cell leaves the codes unchanged; a changed member does not
    perm = g["n3_tris"].copy()
    n0 = int(g["n3_cells"][0, 3])
    perm[:n0] = perm[:n0][::-1]
    assert np.array_equal(cell_list_codes(g["n3_cells"], perm, res, nt), codes)
    perm[0] = (perm[0] + 1) % nt
    assert not np.array_equal(cell_list_codes(g["n3_cells"], perm, res, nt), codes)


def test_window_counts_and_face_pairs_match_the_fixture():
    g = golden("sphere_small.npz")
    res, nt = int(g["res"]), len(g["tris"])
    n4_len = window_counts(g["cell_counts"], res, g["b4_cells"])
    assert np.array_equal(n4_len, g["n4_len"])
    codes = face_pair_codes(g["b4_cells"], g["b4_tris"], g["n4_tris"], n4_len, nt)
    want = np.sort(g["face_pairs"][:, 0].astype(np.int64) * nt + g["face_pairs"][:, 1])
    assert np.array_equal(codes, want)


def test_moving_checkpoint_segments():
    """moving_listener_signal's checkpoint segments: a new one at the first frame at least k steps
    after the current segment's start; every frame belongs to exactly one segment"""
    from pppm_b200.autograd import _segments

    bounds = [0, 15, 30, 45, 60, 75]
    assert _segments(bounds, 30) == [0, 2, 4]
    assert _segments(bounds, 1) == [0, 1, 2, 3, 4]
    assert _segments(bounds, 10 ** 9) == [0]
    assert _segments([0, 7, 9, 40, 41, 100], 20) == [0, 3]
    assert _segments([0, 5], 1) == [0]
