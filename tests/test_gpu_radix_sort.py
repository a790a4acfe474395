"""The library's LSD radix sort (rtnn_sort_pairs, the query-order sort of the pipeline)
against numpy's stable sort -- needs a B200.

Rows never depend on the query order, so a sort that returned a valid but unsorted
permutation would pass every search test; these tests check the order itself: keys come
out non-decreasing in their low `bits` bits, values form the permutation a stable sort
gives (equal keys keep their input order), for 32- and 64-bit keys, sizes around the
2048-key tile, one element, and all-equal keys.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(ctx, keys_np, bits):
    import torch
    n = keys_np.shape[0]
    mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    masked = (keys_np.astype(np.uint64) & mask)
    exp_perm = np.argsort(masked, kind="stable")
    tdt = torch.int64 if keys_np.dtype.itemsize == 8 else torch.int32
    keys = torch.from_numpy(keys_np.view(np.int64 if tdt == torch.int64 else np.int32).copy()).cuda()
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ctx.sort_pairs(keys, vals, bits)
    torch.cuda.synchronize()
    got_keys = keys.cpu().numpy().view(keys_np.dtype)
    got_vals = vals.cpu().numpy()
    assert np.array_equal(np.sort(got_vals), np.arange(n)), "values are not a permutation"
    got_masked = got_keys.astype(np.uint64) & mask
    assert np.all(got_masked[1:] >= got_masked[:-1]), "keys are not sorted"
    assert np.array_equal(got_vals, exp_perm), "not the stable order"
    assert np.array_equal(got_keys, keys_np[exp_perm]), "keys did not move with their values"


@pytest.mark.parametrize("n", [1, 2, 255, 2047, 2048, 2049, 100_003, 1_000_000])
@pytest.mark.parametrize("key_bytes", [4, 8])
def test_random_keys(ctx, n, key_bytes):
    rng = np.random.default_rng(n + key_bytes)
    dt = np.uint64 if key_bytes == 8 else np.uint32
    keys = rng.integers(0, np.iinfo(dt).max, size=n, dtype=dt, endpoint=True)
    _check(ctx, keys, 8 * key_bytes)


@pytest.mark.parametrize("key_bytes,bits", [(4, 12), (4, 27), (8, 36), (8, 61)])
def test_low_bits_only_and_duplicates(ctx, key_bytes, bits):
    """Sorted on the low `bits` bits; the high bits ride along, many equal keys."""
    rng = np.random.default_rng(bits)
    dt = np.uint64 if key_bytes == 8 else np.uint32
    n = 300_001
    keys = rng.integers(0, np.iinfo(dt).max, size=n, dtype=dt, endpoint=True)
    low = rng.integers(0, 1000, size=n).astype(dt)   # few distinct low values
    keys = (keys & ~dt((1 << bits) - 1)) | low
    _check(ctx, keys, bits)


@pytest.mark.parametrize("key_bytes", [4, 8])
def test_all_equal_keys_keep_their_order(ctx, key_bytes):
    dt = np.uint64 if key_bytes == 8 else np.uint32
    keys = np.full(70_001, 0x5A5A5A5A, dtype=dt)
    _check(ctx, keys, 8 * key_bytes)


def test_already_sorted_and_reversed(ctx):
    keys = np.arange(123_457, dtype=np.uint32) * 3
    _check(ctx, keys, 32)
    _check(ctx, keys[::-1].copy(), 32)


def test_rejects_bad_arguments(ctx):
    import torch
    import rtnn_b200
    keys = torch.zeros(10, dtype=torch.int32, device="cuda")
    vals = torch.zeros(10, dtype=torch.int32, device="cuda")
    with pytest.raises(rtnn_b200.RtnnError):
        ctx.sort_pairs(keys, vals, 33)
    with pytest.raises(rtnn_b200.RtnnError):
        ctx.sort_pairs(keys, vals, 0)
