"""GPU test of ae_mpm_radix_sort_keys_noalloc.

That entry point is the cell-key radix sort for callers that cannot allocate GPU memory (an engine
frame loop that runs on memory it reserved up front, work queued while a stream is captured into a
graph, a host whose own pool owns all of HBM).  Its scratch is a fixed array compiled into the
library, shared by every call on a device.  Here it is called through the C ABI on device buffers
this test owns, and its output is compared with a stable CPU sort (numpy's) and with the existing
ae_mpm_radix_sort_keys, on calls in a row, so every call after the first runs on scratch an earlier
one left behind.  The key widths cover every pass plan (1, 2, 3 and 4 passes of at most 8 bits),
and the key counts include ones that are not a multiple of the sort's 2048-key tile.  Keys and
permutation are integers, so the comparison is exact.  The file name makes pytest collect it last.
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


def _cases(rng):
    """(keys, key_bits): 1-, 2-, 3- and 4-pass plans, ragged and tile-multiple counts, full size."""
    mostly_sorted = np.sort(rng.integers(0, 1 << 24, MAX_KEYS, dtype=np.uint64)).astype(np.uint32)
    swaps = rng.integers(0, MAX_KEYS - 1, MAX_KEYS // 16)
    mostly_sorted[swaps], mostly_sorted[swaps + 1] = mostly_sorted[swaps + 1].copy(), mostly_sorted[swaps].copy()
    return [
        (rng.integers(0, 1 << 21, 300001, dtype=np.uint64).astype(np.uint32), 21),
        (mostly_sorted, 24),
        (rng.integers(0, 1 << 8, 4097, dtype=np.uint64).astype(np.uint32), 8),          # 1 pass, ragged
        (rng.integers(0, 1 << 16, 65536, dtype=np.uint64).astype(np.uint32), 16),       # 2 passes, tile multiple
        (rng.integers(0, 1 << 32, 123457, dtype=np.uint64).astype(np.uint32), 32),      # 4 passes, ragged
        (rng.integers(0, 1 << 32, 1, dtype=np.uint64).astype(np.uint32), 32),           # one key
        # bits above key_bits are ignored, as ae_mpm_radix_sort_keys documents
        (rng.integers(0, 1 << 32, 2047, dtype=np.uint64).astype(np.uint32), 12),
    ]


def test_noalloc_sort_matches_a_stable_cpu_sort_on_calls_in_a_row(ctx):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(20261203)
    for keys, bits in _cases(rng):
        got_sorted, got_perm, keys_after = _sort_on_device(ctx, torch, keys, bits)
        masked = keys & np.uint32((1 << bits) - 1 if bits < 32 else 0xFFFFFFFF)
        ref_perm = np.argsort(masked, kind="stable").astype(np.uint32)
        assert np.array_equal(got_perm, ref_perm), (keys.size, bits)
        assert np.array_equal(got_sorted & np.uint32((1 << bits) - 1 if bits < 32 else 0xFFFFFFFF),
                              masked[ref_perm]), (keys.size, bits)
        assert np.array_equal(keys_after, keys)  # the input keys are only read
        alloc_sorted, alloc_perm = ctx.radix_sort(keys, bits)
        assert np.array_equal(got_perm, alloc_perm) and np.array_equal(got_sorted, alloc_sorted)


def test_noalloc_sort_rejects_more_keys_than_its_scratch(ctx):
    torch = pytest.importorskip("torch")
    small = torch.zeros(16, dtype=torch.int32, device="cuda")
    other = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = ctx.lib.ae_mpm_radix_sort_keys_noalloc(ctx.h, small.data_ptr(), MAX_KEYS + 1, 21, other.data_ptr(),
                                                other.data_ptr(), None)
    assert rc == M.EINVAL
    assert "scratch limit" in ctx.lib.ae_mpm_last_error(ctx.h).decode()


def test_noalloc_sort_rejects_overlapping_buffers(ctx):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(3 * 4096, dtype=torch.int32, device="cuda")
    base = buf.data_ptr()
    n = 4096
    # in place (keys = sorted keys), keys overlapping the permutation, and outputs overlapping
    for keys, out, perm in ((base, base, base + 8 * n), (base, base + 4 * n, base + 4 * (n // 2)),
                            (base, base + 4 * n, base + 4 * n + 4 * (n - 1))):
        rc = ctx.lib.ae_mpm_radix_sort_keys_noalloc(ctx.h, keys, n, 8, out, perm, None)
        assert rc == M.EINVAL
        assert "must not overlap" in ctx.lib.ae_mpm_last_error(ctx.h).decode()
    torch.cuda.synchronize()
