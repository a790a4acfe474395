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


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    lib = rtnn_b200.load_library()
    n = lib_max = 1 << 18
    points = torch.zeros((lib_max + 1, 3), dtype=torch.float32, device="cuda")
    out = torch.empty((n + 1, 1), dtype=torch.int32, device="cuda")
    st, msg = _noalloc(lib, points, None, "knn", 1.0, 1, out)
    assert st == 1 and "RTNN_NOALLOC_MAX_POINTS" in msg
