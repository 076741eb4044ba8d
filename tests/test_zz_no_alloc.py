"""GPU test of mb_bitmap_to_rows_noalloc, the row-list entry point for callers
that cannot let the library allocate device memory (hosts that own the whole
device through their own pool, latency-critical callers that cannot afford the
synchronisation an allocation may cause).

It must give exactly what mb_bitmap_to_rows gives (integer output: the
tolerance is zero), on two calls in a row that share its fixed scratch array,
and it must reject sizes beyond its fixed limit before touching the device.
This file is collected last, so a failure here comes after every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from merle_b200 import abi, check, device as D

pytestmark = pytest.mark.gpu


def _random_bitmaps(n: int, seed: int, density: float):
    r = np.random.default_rng(seed)
    W = (n + 31) // 32
    bits = r.random((W, 32)) < density
    words = np.packbits(bits, axis=1, bitorder="little").view(np.uint32).reshape(W)
    unc = words & np.packbits(r.random((W, 32)) < 0.3, axis=1, bitorder="little").view(np.uint32).reshape(W)
    return D.from_host(words), D.from_host(unc)


def _rows(fn, poss, unc, n, cap):
    rows = D.empty(cap, 4, zero=True)
    cnt = D.empty(1, 8, zero=True)
    check(fn(poss.data_ptr(), unc.data_ptr(), n, rows.data_ptr(), cnt.data_ptr(), D.stream_ptr()))
    c = int(D.to_host(cnt, np.uint64)[0])
    return D.to_host(rows, np.uint32)[:c].copy(), c


def test_noalloc_matches_allocating_entry_point(cuda, mb):
    L = mb.lib()
    # the no-allocation entry point runs FIRST, on a size larger than any
    # call before it in this process, and the device's free memory must not
    # move across it (a fallback to an allocating path would show there);
    # then two calls in a row on different inputs: the second must not see
    # the first call's leftovers in the shared scratch array
    warm, wunc = _random_bitmaps(1000, 9, 0.5)
    _rows(L.mb_bitmap_to_rows_noalloc, warm, wunc, 1000, 1032)  # loads the kernels and the array
    for n, seed, density in [(40_000_017, 1, 0.02), (100_003, 2, 0.5)]:
        poss, unc = _random_bitmaps(n, seed, density)
        cap = n + 32
        rows = D.empty(cap, 4, zero=True)
        cnt = D.empty(1, 8, zero=True)
        cuda.cuda.synchronize()
        free0, reserved0 = cuda.cuda.mem_get_info()[0], cuda.cuda.memory_reserved()
        check(L.mb_bitmap_to_rows_noalloc(poss.data_ptr(), unc.data_ptr(), n, rows.data_ptr(), cnt.data_ptr(),
                                          D.stream_ptr()))
        cuda.cuda.synchronize()
        assert cuda.cuda.mem_get_info()[0] == free0 and cuda.cuda.memory_reserved() == reserved0
        gc = int(D.to_host(cnt, np.uint64)[0])
        got = D.to_host(rows, np.uint32)[:gc].copy()
        want, wc = _rows(L.mb_bitmap_to_rows, poss, unc, n, cap)
        assert gc == wc and wc > 0
        np.testing.assert_array_equal(got, want)


def test_noalloc_takes_exactly_its_limit(cuda, mb):
    """nrows == MB_NOALLOC_MAX_ROWS (2^30) is accepted: an all-zero bitmap of
    2^30 rows (128 MiB) gives no row, so a 4-entry output suffices."""
    L = mb.lib()
    limit = 1 << 30
    zero = D.empty(limit // 32, 4, zero=True)
    rows = D.empty(4, 4, zero=True)
    cnt = D.empty(1, 8, zero=True)
    check(L.mb_bitmap_to_rows_noalloc(zero.data_ptr(), None, limit, rows.data_ptr(), cnt.data_ptr(),
                                      D.stream_ptr()))
    assert int(D.to_host(cnt, np.uint64)[0]) == 0


def test_noalloc_rejects_sizes_beyond_its_limit(cuda, mb):
    L = mb.lib()
    limit = 1 << 30
    one = D.empty(4, 4, zero=True)
    cnt = D.empty(1, 8, zero=True)
    st = L.mb_bitmap_to_rows_noalloc(one.data_ptr(), None, limit + 1, one.data_ptr(), cnt.data_ptr(),
                                     D.stream_ptr())
    assert st == abi.MB_ERR_INVALID
    assert b"limit" in L.mb_last_error()
