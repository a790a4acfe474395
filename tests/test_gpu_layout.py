"""Reference-layout output (RTNN_FLAG_REF_LAYOUT + rtnn_layout) through the C ABI -- needs
a B200: rows in the engine's sorted query order holding positions in its sorted point
copy, mapped back with the two permutations, equal the caller-layout rows exactly."""
import numpy as np
import pytest

import rtnn_b200
from rtnn_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _is_perm(a, n):
    return a.shape == (n,) and np.array_equal(np.sort(a.astype(np.int64)), np.arange(n))


@pytest.mark.parametrize("mode,r,k,kw", [("radius", 4.0, 50, {}), ("knn", 3.0, 16, {}),
                                          ("knn", 3.0, 16, {"partition": True})])
def test_single_cloud_ref_layout_maps_back(ctx, mode, r, k, kw):
    p = wl.uniform_cube(30_000, 60.0, seed=11)
    q = wl.uniform_cube(20_000, 60.0, seed=12)
    for queries in (None, q):
        exp = ctx.search(p, queries, mode, r, k, sorted_rows=True, **kw)
        got = ctx.search(p, queries, mode, r, k, sorted_rows=True, ref_layout=True, **kw)
        nq = exp.shape[0]
        po, qo = ctx.layout(p.shape[0], nq)
        assert _is_perm(po, p.shape[0]) and _is_perm(qo, nq)
        assert np.array_equal(rtnn_b200.from_ref_layout(got, po, qo), exp)
        # the rows really are in the engine's order: entries are sorted positions
        assert not np.array_equal(got, exp)


def test_batched_ref_layout_device_buffers(ctx):
    import torch
    p, off = wl.multicloud(n_clouds=40, lo=64, hi=4096, seed=5)
    tp = torch.from_numpy(p).cuda()
    for local in (False, True):
        exp = ctx.search_batched(tp, off, mode="knn", radius=0.2, k=8, sorted_rows=True,
                                 local_indices=local)
        got = ctx.search_batched(tp, off, mode="knn", radius=0.2, k=8, sorted_rows=True,
                                 local_indices=local, ref_layout=True)
        po, qo = ctx.layout(p.shape[0], p.shape[0], device=True)
        po, qo = po.cpu().numpy().astype(np.uint32), qo.cpu().numpy().astype(np.uint32)
        got, exp = got.cpu().numpy(), exp.cpu().numpy()
        if local:   # local positions -> global positions, then caller indices -> local
            cloud = np.searchsorted(off.astype(np.int64), np.arange(p.shape[0]), "right") - 1
            base = off[:-1].astype(np.int64)
            rows_cloud = cloud[qo.astype(np.int64)]
            got = np.where(got >= 0, got + base[rows_cloud][:, None], -1).astype(np.int32)
            back = rtnn_b200.from_ref_layout(got, po, qo)
            back = np.where(back >= 0, back - base[cloud][:, None], -1)
        else:
            back = rtnn_b200.from_ref_layout(got, po, qo)
        assert np.array_equal(back, exp)
        # every cloud's points keep their own block of sorted positions
        cloud_of_pos = np.searchsorted(off.astype(np.int64), np.arange(p.shape[0]), "right") - 1
        cloud_of_pt = np.searchsorted(off.astype(np.int64), po.astype(np.int64), "right") - 1
        assert np.array_equal(cloud_of_pos, cloud_of_pt)


def test_host_batch_with_large_rows_keeps_one_batch_for_the_layout(ctx):
    """A host-buffer batch whose rows pass 256 MB normally runs in sub-batches; with
    RTNN_FLAG_REF_LAYOUT it keeps one batch so that rtnn_layout describes all of it."""
    p, off = wl.multicloud(n_clouds=64, lo=20_000, hi=40_000, seed=6)
    k = 128
    assert p.shape[0] * k * 4 > (256 << 20)
    got = ctx.search_batched(p, off, mode="knn", radius=0.1, k=k, ref_layout=True)
    po, qo = ctx.layout(p.shape[0], p.shape[0])
    exp = ctx.search_batched(p, off, mode="knn", radius=0.1, k=k)
    big = np.iinfo(np.int32).max
    a = np.sort(np.where(exp < 0, big, exp), 1)
    b = rtnn_b200.from_ref_layout(got, po, qo)
    b = np.sort(np.where(b < 0, big, b), 1)
    assert np.array_equal(a, b)
    with pytest.raises(rtnn_b200.RtnnError):   # the sub-batched call left no layout
        ctx.layout(p.shape[0], p.shape[0])


def test_layout_rejects_wrong_sizes(ctx):
    p = wl.uniform_cube(1000, 10.0, seed=1)
    ctx.search(p, None, "knn", 2.0, 4)
    with pytest.raises(rtnn_b200.RtnnError):
        ctx.layout(999, 1000)
