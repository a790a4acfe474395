"""The oracle pinned against the reference's own code and golden vectors (CPU only)."""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_samplepc_golden_rows():
    g = _load("samplepc.json")
    pts = np.asarray(g["points"], dtype=np.float32)
    assert pts.shape == (8, 3)
    for run in g["runs"]:
        got = oracle.bruteforce(pts, None, run["mode"], run["radius"], run["k"])
        assert got.tolist() == run["rows"], run["mode"]
        got_grid = oracle.grid_search(pts, None, run["mode"], run["radius"], run["k"])
        assert got_grid.tolist() == run["rows"]


def test_samplepc_hand_checked():
    g = _load("samplepc.json")
    radius = g["runs"][0]["rows"]
    knn = g["runs"][1]["rows"]
    # radius 2, self included: (5,0,0) and (6,0,0) are 1 apart; (0,0,0) is alone
    assert radius[0][:2] == [0, -1]
    assert sorted(radius[2][:2]) == [2, 4]
    # knn r=10 excludes self: nearest of (0,0,0) are (5,0,0), (6,0,0), (4.99,4.99,0)
    assert knn[0][:3] == [2, 4, 6] and knn[0][3] == -1
    assert 0 not in knn[0] and 2 not in knn[2]


def test_ref_calc_search_size_golden():
    """The oracle's restatement of the reference's shell walk reproduces its masks, and
    the engine's exact box counts never hold fewer points than that walk (it skips the
    twelve edge lines of each shell), so box-count widths are never wider."""
    g = _load("ref_grid.json")
    for grid in g["calc_search_size"]:
        counts = np.asarray(grid["counts_zyx"], dtype=np.uint32)
        need = grid["knn"] + 1
        for c in grid["cells"]:
            cx, cy, cz = c["cell"]
            mask = oracle.ref_shell_mask(counts, cx, cy, cz, grid["cell_size"],
                                         grid["max_width"], grid["knn"])
            assert mask == c["mask"], c
            N = oracle.box_counts(counts, cx, cy, cz, shells=6)
            first = next((s for s, n in enumerate(N) if n >= need), 5)
            assert min(first, 5) <= mask


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_ref_calc_search_size_live():
    rng = np.random.default_rng(11)
    for _ in range(40):
        counts = rng.poisson(rng.uniform(0.1, 2.0), size=(6, 7, 5)).astype(np.uint32)
        knn = int(rng.integers(1, 30))
        cx, cy, cz = int(rng.integers(0, 5)), int(rng.integers(0, 7)), int(rng.integers(0, 6))
        got = oracle.ref_shell_mask(counts, cx, cy, cz, 1.0, 11.0, knn)
        assert got == oracle.ref_calc_search_size(counts, cx, cy, cz, 1.0, 11.0, knn)


def test_morton_golden():
    """The engine's Morton interleave (bit i of x -> 3i, y -> 3i+1, z -> 3i+2) matches
    the reference's MortonCode3 codes."""
    g = _load("ref_grid.json")

    def spread(v):
        r = 0
        for i in range(10):
            r |= ((v >> i) & 1) << (3 * i)
        return r

    for m in g["morton3"]:
        x, y, z = m["xyz"]
        assert spread(x) | (spread(y) << 1) | (spread(z) << 2) == m["code"]


def test_width_from_iter_golden():
    g = _load("ref_grid.json")
    for w in g["width_from_iter"]:
        assert np.float32((2 * w["iter"] + 2) * w["cell"]) == np.float32(w["width"])


@pytest.mark.parametrize("mode,r,k", [("radius", 4.0, 50), ("radius", 4.0, 8), ("knn", 6.0, 5),
                                      ("knn", 3.0, 16)])
def test_grid_oracle_matches_bruteforce(mode, r, k):
    rng = np.random.default_rng(5)
    p = rng.uniform(0, 60, (6000, 3)).astype(np.float32)
    q = rng.uniform(-5, 65, (3000, 3)).astype(np.float32)
    a = oracle.bruteforce(p, q, mode, r, k)
    b = oracle.grid_search(p, q, mode, r, k)
    assert np.array_equal(a, b)


def test_fp32_rows_differ_from_fp64_only_on_boundary_pairs():
    """FP32 and FP64 selections differ only through pairs within ~1 ulp of r."""
    rng = np.random.default_rng(9)
    # quantised coordinates make exact-r distances (and FP32 boundary cases) common
    p = (rng.integers(0, 40, (3000, 3)) * 0.25).astype(np.float32)
    for mode, r in (("radius", 1.0), ("knn", 1.25)):
        a = oracle.bruteforce(p, None, mode, r, 128)
        b = oracle.bruteforce_fp64(p, None, mode, r, 128)
        pairs = oracle.boundary_pairs(p, None, mode, r)
        sa = [set(row[row >= 0].tolist()) for row in a]
        sb = [set(row[row >= 0].tolist()) for row in b]
        diff = set()
        for qi, (x, y) in enumerate(zip(sa, sb)):
            for pi in x ^ y:
                diff.add((qi, pi))
        assert diff == {tuple(v) for v in pairs.tolist()}


def test_ties_break_by_index():
    # a lattice: many points at exactly equal distances
    g = np.stack(np.meshgrid(np.arange(5), np.arange(5), np.arange(5), indexing="ij"), -1)
    p = g.reshape(-1, 3).astype(np.float32)
    rows = oracle.bruteforce(p, None, "knn", 1.5, 4)
    q = 62  # centre (2,2,2): six neighbours at distance 1; the 4 lowest indices win
    d = ((p - p[q]) ** 2).sum(1)
    six = sorted(np.nonzero(d == 1.0)[0].tolist())
    assert rows[q].tolist() == six[:4]


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("mode,r,k", [("radius", 3.0, 50), ("knn", 5.0, 8)])
def test_reference_check_accepts_oracle_and_rejects_planted_mistake(mode, r, k):
    rng = np.random.default_rng(3)
    p = rng.uniform(0, 30, (4000, 3)).astype(np.float32)
    rows = oracle.grid_search(p, None, mode, r, k)
    ok, log = oracle.refcheck(p, None, rows, mode, r, k, 0, 400)
    assert ok, log
    bad = rows.copy()
    q = int(np.argmax((rows >= 0).sum(1)))
    far = int(np.argmax(((p - p[q]) ** 2).sum(1)))
    bad[q, 0] = far  # plant a wrong neighbour in the oracle's output
    ok2, _ = oracle.refcheck(p, None, bad, mode, r, k, q, q + 1)
    assert not ok2


def test_batched_oracle_is_per_cloud():
    rng = np.random.default_rng(4)
    sizes = [50, 0, 300, 7]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    p = rng.uniform(0, 1, (int(off[-1]), 3)).astype(np.float32)
    rows = oracle.grid_search_batched(p, off, mode="knn", r=0.3, k=6)
    for c in range(len(sizes)):
        a, b = int(off[c]), int(off[c + 1])
        if a == b:
            continue
        sub = oracle.bruteforce(p[a:b], None, "knn", 0.3, 6)
        exp = np.where(sub >= 0, sub + a, -1)
        assert np.array_equal(rows[a:b], exp)
    local = oracle.grid_search_batched(p, off, mode="knn", r=0.3, k=6, local=True)
    assert local.max() < max(sizes)


def test_grid_oracle_matches_bruteforce_on_edge_inputs():
    """The grid oracle is the expected result of several GPU tests; on their edge inputs it
    must equal the brute force: lattice points at a 4096 offset with neighbors exactly at
    the radius (r a hair above three steps), coincident points, non-finite and far
    queries (empty rows), a radius whose square is infinite in FP32, K = 1 and 128."""
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(12), indexing="ij"), -1)
    lat = (4096.0 + g.reshape(-1, 3) / 4.0).astype(np.float32)
    lq = np.concatenate([lat[::5], lat[::7] + np.float32(0.125)]).astype(np.float32)
    r = float(np.nextafter(np.float32(0.75), np.float32(1)))
    rng = np.random.default_rng(11)
    dup = np.repeat(rng.uniform(0, 2, (40, 3)).astype(np.float32), 3, axis=0)
    bad_q = np.array([[np.nan, 1, 1], [np.inf, 0, 0], [1e30, 0, 0], [1, 1, 1]], np.float32)
    unit = rng.uniform(0, 1, (500, 3)).astype(np.float32)
    cases = [(lat, lq, r), (dup, None, 0.3), (dup, bad_q, 0.5), (unit, None, 1e20)]
    for p, q, rad in cases:
        for mode in ("radius", "knn"):
            for k in (1, 32, 128):
                a = oracle.bruteforce(p, q, mode, rad, k)
                b = oracle.grid_search(p, q, mode, rad, k)
                assert np.array_equal(a, b), (len(p), mode, rad, k)
    rows = oracle.bruteforce(dup, bad_q, "knn", 0.5, 8)
    assert (rows[:3] == -1).all() and (rows[3] >= 0).any()
