"""Parity of the CUDA search (through the C ABI) with the oracle -- needs a B200.

Index work is compared bit-exactly: each row's neighbor set equals the oracle's, and
with sorted rows the row itself equals the oracle row (order by (FP32 distance, index)).
"""
import json
import os

import numpy as np
import pytest

import oracle
import rtnn_b200
from rtnn_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BIG = np.iinfo(np.int32).max


def as_sets(rows):
    """Rows with their valid entries sorted ascending and -1 kept last."""
    r = np.where(rows < 0, BIG, rows)
    r = np.sort(r, axis=1)
    return np.where(r == BIG, -1, r)


def assert_rows_equal(got, exp, sorted_rows):
    assert got.shape == exp.shape
    if sorted_rows:
        bad = np.nonzero((got != exp).any(1))[0]
    else:
        bad = np.nonzero((as_sets(got) != as_sets(exp)).any(1))[0]
    assert bad.size == 0, (f"{bad.size} rows differ, first {bad[:5].tolist()}: "
                           f"got {got[bad[0]].tolist()} exp {exp[bad[0]].tolist()}")
    # every row: the valid entries come first, then only -1
    valid = got >= 0
    assert (valid[:, :-1] | ~valid[:, 1:]).all()


def test_samplepc_golden(ctx):
    with open(os.path.join(GOLDEN, "samplepc.json")) as f:
        g = json.load(f)
    pts = np.asarray(g["points"], dtype=np.float32)
    for run in g["runs"]:
        got = ctx.search(pts, None, run["mode"], run["radius"], run["k"], sorted_rows=True)
        assert got.tolist() == run["rows"]


@pytest.mark.parametrize("sorted_rows", [False, True])
def test_uniform_radius_full_config(ctx, sorted_rows):
    """Plain fixed-radius search, N = Q = 100,000 uniform in [0,100]^3, r = 4, K = 50."""
    p = wl.uniform_cube(100_000, 100.0, seed=0)
    st = rtnn_b200.Stats()
    got = ctx.search(p, None, "radius", 4.0, 50, sorted_rows=sorted_rows, stats=st)
    exp = oracle.grid_search(p, None, "radius", 4.0, 50)
    assert_rows_equal(got, exp, sorted_rows)
    assert st.n_fallback == 0 and st.n_queries == 100_000


def test_uniform_radius_reference_check(ctx):
    p = wl.uniform_cube(20_000, 60.0, seed=5)
    got = ctx.search(p, None, "radius", 4.0, 50)
    ok, log = oracle.refcheck(p, None, got, "radius", 4.0, 50)
    assert ok, log
    got = ctx.search(p, None, "knn", 4.0, 8)
    ok, log = oracle.refcheck(p, None, got, "knn", 4.0, 8, 0, 2000)
    assert ok, log


@pytest.mark.parametrize("flags", [{}, {"partition": True}])
def test_gmm_knn_small(ctx, flags):
    """KNN K=5, r=10 on a Gaussian mixture with separate uniform queries (scaled)."""
    p, q = wl.gmm(scale=0.05, seed=1)
    got = ctx.search(p, q, "knn", 10.0, 5, sorted_rows=True, **flags)
    exp = oracle.grid_search(p, q, "knn", 10.0, 5)
    assert_rows_equal(got, exp, True)


def test_gmm_knn_full_size_subset(ctx):
    """Full-size KNN config (1e6 points, 1e6 queries): plain and partitioned runs agree
    everywhere, and a seeded subset of rows matches the oracle's brute force."""
    p, q = wl.gmm(seed=1)
    a = ctx.search(p, q, "knn", 10.0, 5, sorted_rows=True)
    st = rtnn_b200.Stats()
    b = ctx.search(p, q, "knn", 10.0, 5, sorted_rows=True, partition=True, stats=st)
    assert np.array_equal(a, b)
    assert st.n_fallback < q.shape[0]
    idx = np.random.default_rng(0).choice(q.shape[0], 1000, replace=False)
    exp = oracle.bruteforce(p, q[idx], "knn", 10.0, 5)
    assert np.array_equal(a[idx], exp)


@pytest.mark.parametrize("mode,r,k", [("knn", 2.0, 16), ("radius", 2.0, 16)])
def test_surfaces_partition(ctx, mode, r, k):
    p = wl.surfaces(scale=0.01, seed=2)
    exp = oracle.grid_search(p, None, mode, r, k)
    for kw in ({}, {"partition": True}):
        st = rtnn_b200.Stats()
        got = ctx.search(p, None, mode, r, k, stats=st, **kw)
        assert_rows_equal(got, exp, False)


def test_sph_lattice_radius_k64(ctx):
    p = wl.sph_lattice(scale=0.0005, seed=4)
    p = wl.sph_step(p, seed=1)
    got = ctx.search(p, None, "radius", 2.0, 64, partition=True)
    exp = oracle.grid_search(p, None, "radius", 2.0, 64)
    assert_rows_equal(got, exp, False)


@pytest.mark.parametrize("k", [1, 2, 31, 32, 33, 64, 100, 128])
def test_k_range(ctx, k):
    p = wl.uniform_cube(8000, 20.0, seed=k)
    for mode in ("radius", "knn"):
        got = ctx.search(p, None, mode, 2.5, k, sorted_rows=True)
        exp = oracle.grid_search(p, None, mode, 2.5, k)
        assert_rows_equal(got, exp, True)


@pytest.mark.parametrize("k", [5, 7, 8, 16, 32, 50, 64])
def test_compiled_k_matches_the_generic_kernels(ctx, k):
    """K in the compiled set runs kernels with K built in (and 16 appended-hit slots);
    another slot count, or a K outside the set (7), runs the generic kernels. Both give the
    oracle's rows, for the tile walk and the one-warp-per-query walk, with many heap
    replacements (about 48 points within r per query)."""
    p = wl.uniform_cube(20_000, 30.0, seed=k)
    base = ctx.tuning().as_dict()
    try:
        for mode in ("radius", "knn"):
            exp = oracle.grid_search(p, None, mode, 2.5, k)
            for qw in (0, 1, 3, 4):
                for slots in (16, 20):
                    ctx.set_tuning(**{**base, "pending_slots": slots, "query_warps": qw})
                    got = ctx.search(p, None, mode, 2.5, k, sorted_rows=True)
                    assert_rows_equal(got, exp, True)
                    got = ctx.search(p, None, mode, 2.5, k)
                    assert_rows_equal(got, exp, False)
    finally:
        ctx.set_tuning(**base)


def test_lattice_ties_break_by_index(ctx):
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(12), indexing="ij"), -1)
    p = g.reshape(-1, 3).astype(np.float32)
    for mode, r, k in (("knn", 1.5, 4), ("knn", 2.0, 10), ("radius", 1.5, 5), ("radius", 1.0001, 3)):
        got = ctx.search(p, None, mode, r, k, sorted_rows=True)
        exp = oracle.bruteforce(p, None, mode, r, k)
        assert_rows_equal(got, exp, True)


def test_points_exactly_at_radius_are_excluded(ctx):
    p = np.array([[0, 0, 0], [2, 0, 0], [0, 2, 0], [1.9999999, 0, 0], [0, 0, -2]], np.float32)
    got = ctx.search(p, None, "radius", 2.0, 8, sorted_rows=True)
    exp = oracle.bruteforce(p, None, "radius", 2.0, 8)
    assert_rows_equal(got, exp, True)
    assert 1 not in got[0] and 3 in got[0]


def test_duplicates(ctx):
    p = np.zeros((300, 3), np.float32)
    p[200:] = 0.5
    knn = ctx.search(p, None, "knn", 1.0, 8)
    # coincident points are excluded in KNN: the 200 zeros only see the 100 halves
    assert (knn[:200] >= 200).all()
    rad = ctx.search(p, None, "radius", 1.0, 8, sorted_rows=True)
    exp = oracle.bruteforce(p, None, "radius", 1.0, 8)
    assert_rows_equal(rad, exp, True)


def test_empty_inputs(ctx):
    p = wl.uniform_cube(100, 10.0, seed=1)
    empty = np.zeros((0, 3), np.float32)
    out = ctx.search(empty, p, "radius", 1.0, 4)
    assert out.shape == (100, 4) and (out == -1).all()
    out = ctx.search(p, empty, "knn", 1.0, 4)
    assert out.shape == (0, 4)


def test_far_and_nonfinite_queries(ctx):
    p = wl.uniform_cube(2000, 10.0, seed=2)
    q = np.array([[1e6, 1e6, 1e6], [-1e30, 0, 0], [np.nan, 1, 1], [np.inf, 0, 0], [5, 5, 5]],
                 np.float32)
    got = ctx.search(p, q, "knn", 2.0, 6, sorted_rows=True)
    assert (got[:4] == -1).all()
    exp = oracle.bruteforce(p, q[4:], "knn", 2.0, 6)
    assert np.array_equal(got[4:], exp)


def test_nonfinite_query_rows_are_written(ctx):
    """Rows of queries that cannot be searched (NaN or infinite coordinates) are filled
    with -1 by the search itself, whatever the output buffer held before."""
    import torch
    p = wl.uniform_cube(3000, 10.0, seed=3)
    q = np.array([[np.nan, 1, 1], [1, np.inf, 1], [5, 5, 5], [1, 1, -np.inf]], np.float32)
    tp, tq = torch.from_numpy(p).cuda(), torch.from_numpy(q).cuda()
    for mode in ("knn", "radius"):
        for part in (False, True):
            out = torch.full((4, 6), 7, dtype=torch.int32, device="cuda")
            ctx.search(tp, tq, mode, 2.0, 6, partition=part, sorted_rows=True, out=out)
            got = out.cpu().numpy()
            assert (got[[0, 1, 3]] == -1).all(), got
            assert np.array_equal(got[2], oracle.bruteforce(p, q[2:3], mode, 2.0, 6)[0])


def test_invalid_arguments(ctx):
    p = wl.uniform_cube(10, 1.0, seed=0)
    with pytest.raises(rtnn_b200.RtnnError) as e:
        ctx.search(p, None, "knn", 1.0, 0)
    assert e.value.code == "RTNN_ERR_UNSUPPORTED_K"
    with pytest.raises(rtnn_b200.RtnnError) as e:
        ctx.search(p, None, "knn", 1.0, 129)
    assert e.value.code == "RTNN_ERR_UNSUPPORTED_K"
    for bad_r in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(rtnn_b200.RtnnError) as e:
            ctx.search(p, None, "radius", bad_r, 4)
        assert e.value.code == "RTNN_ERR_INVALID_ARGUMENT"
    fresh = rtnn_b200.Context(0)
    with pytest.raises(rtnn_b200.RtnnError) as e:
        fresh.search(p, None, "knn", 1.0, 4, learned=True)
    assert e.value.code == "RTNN_ERR_NO_MODEL"
    fresh.close()
    # the context stays usable after rejected calls
    assert ctx.search(p, None, "radius", 1.0, 4).shape == (10, 4)


def test_device_pointers(ctx):
    import torch
    p, q = wl.gmm(scale=0.02, seed=7)
    tp = torch.from_numpy(p).cuda()
    tq = torch.from_numpy(q).cuda()
    out = ctx.search(tp, tq, "knn", 10.0, 5, sorted_rows=True)
    assert out.is_cuda and out.dtype == torch.int32
    exp = oracle.grid_search(p, q, "knn", 10.0, 5)
    assert np.array_equal(out.cpu().numpy(), exp)


def test_unaligned_inputs(ctx):
    """Inputs starting off a 16-byte boundary take the scalar load path."""
    import torch
    p = wl.uniform_cube(5001, 20.0, seed=3)
    buf = torch.from_numpy(np.concatenate([np.zeros(1, np.float32), p.ravel()])).cuda()
    tp = buf[1:].view(-1, 3)
    assert tp.data_ptr() % 16 != 0
    out = ctx.search(tp, None, "radius", 2.0, 12, sorted_rows=True)
    exp = oracle.grid_search(p, None, "radius", 2.0, 12)
    assert np.array_equal(out.cpu().numpy(), exp)


def test_batched_matches_per_cloud_oracle(ctx):
    p, off = wl.multicloud(n_clouds=64, lo=16, hi=4000, seed=3)
    for local in (False, True):
        st = rtnn_b200.Stats()
        got = ctx.search_batched(p, off, mode="knn", radius=0.2, k=32, local_indices=local,
                                 stats=st)
        exp = oracle.grid_search_batched(p, off, mode="knn", r=0.2, k=32, local=local)
        assert_rows_equal(got, exp, False)
        assert st.n_clouds == 64


def test_batched_host_buffers_in_sub_batches(ctx):
    """A host-buffer batch whose rows exceed 256 MB runs as sub-batches of whole clouds with
    the downloads overlapped: same rows as the device-pointer call (one batch), stats summed."""
    import torch
    p, off = wl.multicloud(n_clouds=64, lo=8000, hi=40000, seed=21)
    k = 64
    assert p.shape[0] * k * 4 >= 256 << 20
    tp = torch.from_numpy(p).cuda()
    for kw in ({}, {"partition": True}):
        dev = ctx.search_batched(tp, off, mode="knn", radius=0.2, k=k, sorted_rows=True, **kw)
        st = rtnn_b200.Stats()
        host = ctx.search_batched(p, off, mode="knn", radius=0.2, k=k, sorted_rows=True, stats=st,
                                  **kw)
        assert np.array_equal(host, dev.cpu().numpy())
        assert st.n_queries == p.shape[0] and st.n_clouds == 64 and st.ms_total > 0
    anyk = ctx.search_batched(p, off, mode="radius", radius=0.2, k=k, any_k=True)
    full = ctx.search_batched(tp, off, mode="radius", radius=0.2, k=k).cpu().numpy()
    assert np.array_equal((anyk >= 0).sum(1), (full >= 0).sum(1))


def test_batched_separate_queries_and_empty_clouds(ctx):
    rng = np.random.default_rng(8)
    psz = [100, 0, 50, 300, 1]
    qsz = [20, 5, 0, 40, 3]
    po = np.concatenate([[0], np.cumsum(psz)]).astype(np.uint64)
    qo = np.concatenate([[0], np.cumsum(qsz)]).astype(np.uint64)
    p = rng.uniform(0, 1, (int(po[-1]), 3)).astype(np.float32)
    q = rng.uniform(0, 1, (int(qo[-1]), 3)).astype(np.float32)
    for mode in ("knn", "radius"):
        got = ctx.search_batched(p, po, q, qo, mode=mode, radius=0.3, k=7, partition=True)
        exp = oracle.grid_search_batched(p, po, q, qo, mode=mode, r=0.3, k=7)
        assert_rows_equal(got, exp, False)


def test_plan_graph_replay(ctx):
    import torch
    p, off = wl.multicloud(n_clouds=32, lo=64, hi=3000, seed=5)
    tp = torch.from_numpy(p).cuda()
    exp = oracle.grid_search_batched(p, off, mode="knn", r=0.2, k=16)
    for use_graph in (False, True):
        plan = ctx.plan(off, mode="knn", radius=0.2, k=16, use_graph=use_graph)
        for _ in range(3):
            out = plan.execute(tp)
            assert_rows_equal(out.cpu().numpy(), exp, False)
        # new point data of the same shape through the same graph
        p2 = (p * np.float32(0.9) + np.float32(0.05)).astype(np.float32)
        tp.copy_(torch.from_numpy(p2))
        out = plan.execute(tp)
        exp2 = oracle.grid_search_batched(p2, off, mode="knn", r=0.2, k=16)
        assert_rows_equal(out.cpu().numpy(), exp2, False)
        tp.copy_(torch.from_numpy(p))
        plan.close()


@pytest.mark.parametrize("use_graph", [False, True])
def test_plan_keep_order_time_steps(ctx, use_graph):
    """KEEP_ORDER plans sort the queries on the first execute only and reuse that order
    (no query keys, no sort) while the points move: rows stay exact through small steps,
    through a shuffle of the positions inside every cloud (the kept order then means
    nothing), and after resort(), which sorts once more."""
    import ctypes
    import torch
    p, off = wl.multicloud(n_clouds=24, lo=64, hi=3000, seed=9)
    rng = np.random.default_rng(4)
    for flags in ({}, {"partition": True}):
        cur = p.copy()
        tp = torch.from_numpy(cur).cuda()
        plan = ctx.plan(off, mode="knn", radius=0.2, k=16, use_graph=use_graph,
                        sorted_rows=True, keep_order=True, **flags)
        launches = []
        for step in range(4):
            st = rtnn_b200.Stats()
            out = plan.execute(tp, stats=st)
            launches.append(st.n_launches)
            exp = oracle.grid_search_batched(cur, off, mode="knn", r=0.2, k=16)
            assert np.array_equal(out.cpu().numpy(), exp), f"step {step}"
            if step == 1:
                for c in range(len(off) - 1):
                    a, b = int(off[c]), int(off[c + 1])
                    cur[a:b] = cur[a:b][rng.permutation(b - a)]
            else:
                cur = (cur + rng.normal(0.0, 0.005, cur.shape)).astype(np.float32)
            tp.copy_(torch.from_numpy(cur))
        assert launches[1] < launches[0] and launches[1] == launches[2] == launches[3]
        plan.resort()
        st = rtnn_b200.Stats()
        out = plan.execute(tp, stats=st)
        assert st.n_launches == launches[0]
        exp = oracle.grid_search_batched(cur, off, mode="knn", r=0.2, k=16)
        assert np.array_equal(out.cpu().numpy(), exp)
        plan.close()
    # the flag belongs to plans: a one-shot search rejects it
    lib = rtnn_b200.load_library()
    q = wl.uniform_cube(10, 1.0, seed=0)
    res = np.empty((10, 4), np.int32)
    st = lib.rtnn_search(ctx._h, q.ctypes.data_as(ctypes.c_void_p), 10, None, 10,
                         rtnn_b200.KNN, 1.0, 4, rtnn_b200.FLAG_KEEP_ORDER,
                         res.ctypes.data_as(ctypes.c_void_p), None)
    assert st != 0


def test_fp64_disagreement_is_only_boundary_pairs(ctx):
    rng = np.random.default_rng(9)
    p = (rng.integers(0, 40, (3000, 3)) * 0.25).astype(np.float32)
    for mode, r in (("radius", 1.0), ("knn", 1.25)):
        got = ctx.search(p, None, mode, r, 128)
        ref64 = oracle.bruteforce_fp64(p, None, mode, r, 128)
        pairs = {tuple(v) for v in oracle.boundary_pairs(p, None, mode, r).tolist()}
        diff = set()
        for qi in range(p.shape[0]):
            a = set(got[qi][got[qi] >= 0].tolist())
            b = set(ref64[qi][ref64[qi] >= 0].tolist())
            diff |= {(qi, x) for x in a ^ b}
        assert diff == pairs


@pytest.mark.parametrize("ratio", [0.0, 0.01, 1.0, 1e9])
def test_walk_modes_give_identical_rows(ctx, ratio):
    """Shared candidate stream (ratio 0 or huge) and per-lane walk (tiny ratio) agree
    with the oracle row for row, in every mode and with the partition on."""
    base = ctx.tuning().as_dict()
    try:
        ctx.set_tuning(**{**base, "lane_walk_ratio": ratio})
        p, off = wl.multicloud(n_clouds=24, lo=64, hi=6000, seed=9)
        got = ctx.search_batched(p, off, mode="knn", radius=0.2, k=32, sorted_rows=True,
                                 partition=True)
        assert np.array_equal(got, oracle.grid_search_batched(p, off, mode="knn", r=0.2, k=32))
        u = wl.uniform_cube(30_000, 40.0, seed=4)
        for mode in ("radius", "knn"):
            got = ctx.search(u, None, mode, 3.0, 40, sorted_rows=True)
            assert np.array_equal(got, oracle.grid_search(u, None, mode, 3.0, 40))
    finally:
        ctx.set_tuning(**base)


@pytest.mark.parametrize("slots", [8, 12, 32, 256])
def test_pending_slots_give_identical_rows(ctx, slots):
    """Few slots force many merges of appended hits into the kept K (some lanes at exactly
    K kept when another lane's column fills); many slots merge once. Rows match the
    oracle either way, for small and large K, with the partition on and off."""
    base = ctx.tuning().as_dict()
    try:
        ctx.set_tuning(**{**base, "pending_slots": slots})
        u = wl.uniform_cube(20_000, 40.0, seed=1)
        for mode, k in (("knn", 5), ("knn", 64), ("radius", 7), ("radius", 128)):
            exp = oracle.grid_search(u, None, mode, 3.0, k)
            for part in (False, True):
                got = ctx.search(u, None, mode, 3.0, k, partition=part)
                assert_rows_equal(got, exp, sorted_rows=False)
        p, off = wl.multicloud(n_clouds=16, lo=64, hi=4000, seed=3)
        got = ctx.search_batched(p, off, mode="knn", radius=0.2, k=32, sorted_rows=True,
                                 partition=True)
        assert np.array_equal(got, oracle.grid_search_batched(p, off, mode="knn", r=0.2, k=32))
    finally:
        ctx.set_tuning(**base)


@pytest.mark.parametrize("qw", [1, 2, 3, 4])
@pytest.mark.parametrize("k", [1, 5, 32, 64, 96, 128])
def test_query_warps_match_oracle(ctx, k, qw):
    """One warp per query (query_warps 1: every pass; 2: escalation passes only; K > 64
    falls back to the tile walk) and the lane walk (3: first pass, one warp per query for the
    escalations; 4: every pass): rows equal the oracle's, sorted and as sets, with the
    partition off and on (escalation passes included), in batched clouds, and with ANY_K."""
    base = ctx.tuning().as_dict()
    try:
        ctx.set_tuning(**{**base, "query_warps": qw})
        u = wl.uniform_cube(20_000, 40.0, seed=5)
        for mode in ("knn", "radius"):
            exp = oracle.grid_search(u, None, mode, 3.0, k)
            assert np.array_equal(ctx.search(u, None, mode, 3.0, k, sorted_rows=True), exp)
            for part in (False, True):
                assert_rows_equal(ctx.search(u, None, mode, 3.0, k, partition=part), exp, False)
            anyk = ctx.search(u, None, mode, 3.0, k, any_k=True)
            n_exp = (exp >= 0).sum(1)
            assert np.array_equal((anyk >= 0).sum(1), n_exp)
            for qi in range(0, u.shape[0], 211):
                g = anyk[qi][anyk[qi] >= 0]
                assert len(set(g.tolist())) == len(g)
        p, off = wl.multicloud(n_clouds=16, lo=64, hi=4000, seed=8)
        got = ctx.search_batched(p, off, mode="knn", radius=0.2, k=min(k, 32), sorted_rows=True,
                                 partition=True)
        assert np.array_equal(got, oracle.grid_search_batched(p, off, mode="knn", r=0.2,
                                                              k=min(k, 32)))
        q = np.array([[np.nan, 1, 1], [20, 20, 20], [1e9, 0, 0]], np.float32)
        got = ctx.search(u, q, "knn", 3.0, k, sorted_rows=True)
        assert (got[[0, 2]] == -1).all()
        assert np.array_equal(got[1], oracle.bruteforce(u, q[1:2], "knn", 3.0, k)[0])
    finally:
        ctx.set_tuning(**base)


@pytest.mark.parametrize("cell_ratio", [1.0 / 3.0, 0.5, 1.0])
def test_clipped_rows_keep_points_at_the_radius(ctx, cell_ratio):
    """The walks skip cell rows (and the ends of rows) that lie entirely farther than the
    search width from the query box. Lattice points far from the origin (4096 + i / 4,
    where the cell map rounds most) sit on or next to cell boundaries, and r is a hair above
    three lattice steps, so many neighbors lie exactly at the edge of the ball: every
    kernel choice, with the partition off and on, must return the oracle's rows."""
    base = ctx.tuning().as_dict()
    g = np.stack(np.meshgrid(np.arange(24), np.arange(24), np.arange(24), indexing="ij"), -1)
    p = (4096.0 + g.reshape(-1, 3) / 4.0).astype(np.float32)
    q = np.concatenate([p[::7], p[::11] + np.float32(0.125)]).astype(np.float32)
    r = float(np.nextafter(np.float32(0.75), np.float32(1)))
    try:
        for qw in (0, 1, 2, 3, 4):
            ctx.set_tuning(**{**base, "cell_ratio": cell_ratio, "points_per_cell": 0.0,
                              "query_warps": qw})
            for mode, k in (("knn", 32), ("radius", 128), ("knn", 20)):
                exp = oracle.grid_search(p, q, mode, r, k)
                for part in (False, True):
                    got = ctx.search(p, q, mode, r, k, partition=part, sorted_rows=True)
                    assert_rows_equal(got, exp, True)
                    # unsorted rows: the K kept among lattice ties at equal distances
                    got = ctx.search(p, q, mode, r, k, partition=part)
                    assert_rows_equal(got, exp, False)
    finally:
        ctx.set_tuning(**base)


def test_clip_off_for_widths_beyond_the_grid(ctx):
    """A radius of 1e20 over a unit cloud with cells of a few hundredths (min_cell_ratio
    1e-25 lets the cells stay small): the width is ~1e21 cells, where squares overflow
    FP32, so the row clip must switch itself off and walk every row. r * r is infinite,
    so every point qualifies and the rows are the K nearest."""
    base = ctx.tuning().as_dict()
    u = wl.uniform_cube(2000, 1.0, seed=3)
    try:
        for qw in (0, 1, 4):
            ctx.set_tuning(**{**base, "cell_ratio": 0.125, "min_cell_ratio": 1e-25,
                              "points_per_cell": 0.125, "query_warps": qw})
            for mode, k in (("radius", 128), ("knn", 32), ("knn", 64)):
                exp = oracle.bruteforce(u, None, mode, 1e20, k)
                got = ctx.search(u, None, mode, 1e20, k, sorted_rows=True)
                assert_rows_equal(got, exp, True)
    finally:
        ctx.set_tuning(**base)


def test_bounded_wait_reports_timeout_and_context_survives(ctx):
    """A device-side wait that can never be satisfied (a scan predecessor nobody
    publishes) gives up after its limit and reports RTNN_ERR_DEVICE_TIMEOUT; the context
    and the GPU stay usable."""
    import time
    lib = rtnn_b200.load_library()
    t0 = time.time()
    st = lib.rtnn_selftest_wait_timeout(ctx.handle)
    assert st == 5, lib.rtnn_last_error(ctx.handle)   # RTNN_ERR_DEVICE_TIMEOUT
    assert time.time() - t0 < 60
    assert b"gave up" in lib.rtnn_last_error(ctx.handle)
    p = wl.uniform_cube(5000, 20.0, seed=1)
    got = ctx.search(p, None, "radius", 2.0, 16, sorted_rows=True)
    assert np.array_equal(got, oracle.grid_search(p, None, "radius", 2.0, 16))


@pytest.mark.parametrize("mode", ["radius", "knn"])
def test_any_k_returns_k_qualifying_points(ctx, mode):
    """RTNN_FLAG_ANY_K: every row holds min(K, #qualifying) distinct qualifying points
    (the reference's radius semantics); which ones is unspecified."""
    p = wl.uniform_cube(30_000, 30.0, seed=6)
    k, r = 12, 2.5
    full = oracle.grid_search(p, None, mode, r, 128)
    got = ctx.search(p, None, mode, r, k, any_k=True)
    n_q = (full >= 0).sum(1)
    assert np.array_equal((got >= 0).sum(1), np.minimum(n_q, k))
    for qi in range(0, p.shape[0], 97):
        g = got[qi][got[qi] >= 0]
        assert len(set(g.tolist())) == len(g)
        assert set(g.tolist()) <= set(full[qi][full[qi] >= 0].tolist())
