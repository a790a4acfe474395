"""Host side of the reference-layout output (RTNN_FLAG_REF_LAYOUT): remapping rows
written in the engine's order back to the caller's order (no GPU).

The reference returns indices into its Morton-sorted copy of the points, in rows that
follow its partitioned query arrays (sort.cpp:378-386,612,626; search.cpp:43-53); a
reference-layout search here returns the same kind of buffer for the engine's own sorted
orders, and rtnn_b200.from_ref_layout maps it back with the two permutations.
"""
import numpy as np

import rtnn_b200


def test_from_ref_layout_inverts_a_planted_layout():
    rng = np.random.default_rng(0)
    n_pts, n_q, k = 500, 300, 7
    caller = rng.integers(-1, n_pts, size=(n_q, k)).astype(np.int32)
    caller[rng.random((n_q, k)) < 0.2] = -1
    point_order = rng.permutation(n_pts).astype(np.uint32)   # sorted position -> caller index
    query_order = rng.permutation(n_q).astype(np.uint32)     # row -> caller query
    pos_of = np.empty(n_pts, np.int64)
    pos_of[point_order] = np.arange(n_pts)
    ref_rows = np.where(caller >= 0, pos_of[np.where(caller >= 0, caller, 0)], -1)
    ref_rows = ref_rows[query_order].astype(np.int32)
    back = rtnn_b200.from_ref_layout(ref_rows, point_order, query_order)
    assert back.dtype == np.int32
    assert np.array_equal(back, caller)


def test_from_ref_layout_keeps_empty_rows():
    rows = np.full((4, 3), -1, np.int32)
    back = rtnn_b200.from_ref_layout(rows, np.arange(10, dtype=np.uint32),
                                     np.array([3, 1, 0, 2], np.uint32))
    assert (back == -1).all()
