"""GPU test of ae_mpm_radix_sort_keys_noalloc.

That entry point is the cell-key radix sort for callers that cannot allocate GPU memory (an engine
frame loop that runs on memory it reserved up front, work queued while a stream is captured into a
graph, a host whose own pool owns all of HBM).  Its scratch is a fixed array compiled into the
library, shared by every call on a device.  Here it is called through the C ABI on device buffers
this test owns, and its output is compared with the existing ae_mpm_radix_sort_keys on two calls
in a row, so the second call runs on scratch the first one left behind.  Keys and permutation are
integers, so the comparison is exact.  The file name makes pytest collect it last.
"""
import numpy as np
import pytest

import ae_mpm as M

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20  # AE_MPM_NOALLOC_MAX_KEYS


def _sort_on_device(ctx, torch, keys, bits):
    d_keys = torch.from_numpy(keys.view(np.int32).copy()).cuda()
    d_sorted = torch.empty_like(d_keys)
    d_perm = torch.empty_like(d_keys)
    torch.cuda.synchronize()
    rc = ctx.lib.ae_mpm_radix_sort_keys_noalloc(ctx.h, d_keys.data_ptr(), keys.size, bits, d_sorted.data_ptr(),
                                                d_perm.data_ptr(), None)
    ctx.check(rc)
    torch.cuda.synchronize()
    view = lambda t: t.cpu().numpy().view(np.uint32)  # noqa: E731
    return view(d_sorted), view(d_perm), view(d_keys)


def test_noalloc_sort_matches_the_allocating_sort_on_two_calls(ctx):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(20261203)
    first = rng.integers(0, 1 << 21, 300001, dtype=np.uint64).astype(np.uint32)
    second = np.sort(rng.integers(0, 1 << 24, MAX_KEYS, dtype=np.uint64)).astype(np.uint32)
    swaps = rng.integers(0, MAX_KEYS - 1, MAX_KEYS // 16)
    second[swaps], second[swaps + 1] = second[swaps + 1].copy(), second[swaps].copy()
    for keys, bits in ((first, 21), (second, 24)):
        got_sorted, got_perm, keys_after = _sort_on_device(ctx, torch, keys, bits)
        ref_sorted, ref_perm = ctx.radix_sort(keys, bits)
        assert np.array_equal(got_perm, ref_perm)
        assert np.array_equal(got_sorted, ref_sorted)
        assert np.array_equal(keys_after, keys)  # the input keys are only read


def test_noalloc_sort_rejects_more_keys_than_its_scratch(ctx):
    torch = pytest.importorskip("torch")
    small = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = ctx.lib.ae_mpm_radix_sort_keys_noalloc(ctx.h, small.data_ptr(), MAX_KEYS + 1, 21, small.data_ptr(),
                                                small.data_ptr(), None)
    assert rc == M.EINVAL
    assert "scratch limit" in ctx.lib.ae_mpm_last_error(ctx.h).decode()
