"""rtnn_search_noalloc -- the search entry point for callers that cannot allocate device
memory (a host that owns all device memory through its own pool, a real-time loop that
cannot afford cudaMalloc's implicit device synchronisation, code running during a global
stream capture). Called through the C ABI, it must return the same neighbor sets as
rtnn_search (flags 0) on consecutive calls, although every call reuses the same fixed
scratch array and keeps none of the previous call's state.

This file is collected last on purpose: a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

import rtnn_b200
from rtnn_b200 import workloads as wl

pytestmark = pytest.mark.gpu

BIG = np.iinfo(np.int32).max


def _sets(rows):
    r = np.where(rows < 0, BIG, rows)
    return np.sort(r, axis=1)


def _noalloc(lib, points, queries, mode, radius, k, out):
    err = ctypes.create_string_buffer(512)
    st = lib.rtnn_search_noalloc(
        ctypes.c_void_p(points.data_ptr()), points.shape[0],
        ctypes.c_void_p(queries.data_ptr()) if queries is not None else None,
        points.shape[0] if queries is None else queries.shape[0],
        rtnn_b200._mode(mode), float(radius), int(k), ctypes.c_void_p(out.data_ptr()), None,
        err, len(err))
    return st, err.value.decode()


def test_noalloc_matches_rtnn_search_on_two_calls_in_a_row():
    import torch
    lib = rtnn_b200.load_library()
    ctx = rtnn_b200.Context(0)
    p1 = torch.from_numpy(wl.uniform_cube(60_000, 60.0, seed=0)).cuda()
    p2, q2 = wl.gmm(scale=0.04, seed=1)
    p2, q2 = torch.from_numpy(p2).cuda(), torch.from_numpy(q2).cuda()
    calls = [(p1, None, "radius", 4.0, 50), (p2, q2, "knn", 10.0, 5)]
    for points, queries, mode, radius, k in calls:
        nq = points.shape[0] if queries is None else queries.shape[0]
        out = torch.full((nq, k), 7, dtype=torch.int32, device="cuda")
        st, msg = _noalloc(lib, points, queries, mode, radius, k, out)
        assert st == 0, msg
        exp = ctx.search(points, queries, mode, radius, k)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(_sets(got), _sets(exp.cpu().numpy())), mode
    ctx.close()


MAX_POINTS = 1 << 18    # RTNN_NOALLOC_MAX_POINTS
MAX_QUERIES = 1 << 18   # RTNN_NOALLOC_MAX_QUERIES


@pytest.mark.parametrize("mode,radius,k", [("radius", 2.0, 32), ("knn", 2.0, 16)])
def test_noalloc_at_its_documented_maximum(mode, radius, k):
    """Exactly RTNN_NOALLOC_MAX_POINTS points and RTNN_NOALLOC_MAX_QUERIES separate
    queries (density 1 per unit cell, about 33 points within r): the fixed layout fits the
    array and the rows equal rtnn_search's."""
    import torch
    lib = rtnn_b200.load_library()
    ctx = rtnn_b200.Context(0)
    p = torch.from_numpy(wl.uniform_cube(MAX_POINTS, 64.0, seed=7)).cuda()
    q = torch.from_numpy(wl.uniform_cube(MAX_QUERIES, 64.0, seed=8)).cuda()
    assert p.shape[0] == MAX_POINTS and q.shape[0] == MAX_QUERIES
    out = torch.full((MAX_QUERIES, k), 7, dtype=torch.int32, device="cuda")
    st, msg = _noalloc(lib, p, q, mode, radius, k, out)
    assert st == 0, msg
    exp = ctx.search(p, q, mode, radius, k)
    torch.cuda.synchronize()
    assert np.array_equal(_sets(out.cpu().numpy()), _sets(exp.cpu().numpy()))
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    lib = rtnn_b200.load_library()
    points = torch.zeros((MAX_POINTS + 1, 3), dtype=torch.float32, device="cuda")
    out = torch.empty((MAX_POINTS + 1, 1), dtype=torch.int32, device="cuda")
    st, msg = _noalloc(lib, points, None, "knn", 1.0, 1, out)
    assert st == 1 and "RTNN_NOALLOC_MAX_POINTS" in msg
    # the query limit on its own: few points, one query too many
    few = torch.zeros((16, 3), dtype=torch.float32, device="cuda")
    queries = torch.zeros((MAX_QUERIES + 1, 3), dtype=torch.float32, device="cuda")
    out.fill_(5)
    torch.cuda.synchronize()
    st, msg = _noalloc(lib, few, queries, "knn", 1.0, 1, out)
    assert st == 1 and "RTNN_NOALLOC_MAX_QUERIES" in msg
    torch.cuda.synchronize()
    assert int(out.min()) == 5 and int(out.max()) == 5   # rejected before any work


def test_noalloc_beside_a_global_mode_capture():
    """One thread captures a CUDA graph in global mode while another searches on a
    non-blocking stream: the search succeeds and the capture stays valid."""
    import threading
    import torch
    lib = rtnn_b200.load_library()
    ctx = rtnn_b200.Context(0)
    p = torch.from_numpy(wl.uniform_cube(20_000, 30.0, seed=9)).cuda()
    out = torch.empty((20_000, 8), dtype=torch.int32, device="cuda")
    st, msg = _noalloc(lib, p, None, "knn", 2.0, 8, out)   # first call: set-up, no capture
    assert st == 0, msg
    torch.cuda.synchronize()
    x = torch.zeros(1024, device="cuda")
    graph = torch.cuda.CUDAGraph()
    capturing, searched = threading.Event(), threading.Event()
    result = {}

    s = torch.cuda.Stream()   # torch's pool streams are created non-blocking

    def search_thread():
        capturing.wait(30)
        err = ctypes.create_string_buffer(512)
        result["st"] = lib.rtnn_search_noalloc(
            ctypes.c_void_p(p.data_ptr()), p.shape[0], None, 0, rtnn_b200.KNN, 2.0, 8,
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream), err, len(err))
        result["msg"] = err.value.decode()
        searched.set()

    t = threading.Thread(target=search_thread)
    t.start()
    with torch.cuda.graph(graph, capture_error_mode="global"):
        x.add_(1.0)
        capturing.set()
        searched.wait(60)
        x.mul_(2.0)
    t.join(60)
    assert result.get("st") == 0, result.get("msg")
    graph.replay()
    torch.cuda.synchronize()
    assert float(x.min()) == 2.0 and float(x.max()) == 2.0
    exp = ctx.search(p, None, "knn", 2.0, 8)
    torch.cuda.synchronize()
    assert np.array_equal(_sets(out.cpu().numpy()), _sets(exp.cpu().numpy()))
    ctx.close()
