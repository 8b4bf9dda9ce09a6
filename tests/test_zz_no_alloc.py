"""The allocation-free radix sort (hr_radix_sort_pairs_noalloc).

Some callers cannot allocate device memory once their loop is running: a renderer or a
serving process that reserves its whole HBM budget at start-up must not call cudaMalloc
per frame, because an allocation can stall the device or fail under memory pressure.
For them the library offers one sort that needs no context and allocates nothing; its
scratch is a static per-GPU array.  This test calls it through the C-ABI twice in a row
and checks each result against the allocating entry point, bit for bit (the tolerance of
every integer parity test here).  The file sorts last so that a run stopping at the
first failure has already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sort_allocating(engine, keys, vals, bits):
    import torch
    tk = torch.from_numpy(keys.view(np.int32)).cuda()
    tv = torch.from_numpy(vals.view(np.int32)).cuda()
    torch.cuda.synchronize()
    engine.radix_sort_pairs_device(tk, tv, keys.size, bits)
    return tk.cpu().numpy().view(np.uint32), tv.cpu().numpy().view(np.uint32)


def _sort_noalloc(hrlib, keys, vals, bits):
    import torch
    tk = torch.from_numpy(keys.view(np.int32)).cuda()
    tv = torch.from_numpy(vals.view(np.int32)).cuda()
    stream = torch.cuda.current_stream()
    st = hrlib.hr_radix_sort_pairs_noalloc(C.c_void_p(stream.cuda_stream), C.c_void_p(tk.data_ptr()),
                                           C.c_void_p(tv.data_ptr()), keys.size, bits)
    assert st == 0
    torch.cuda.synchronize()
    return tk.cpu().numpy().view(np.uint32), tv.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_twice(hrlib, engine):
    rng = np.random.default_rng(2024)
    # two calls in a row: the second is smaller and uses fewer bits, so stale scratch
    # left by the first call would show up as a mismatch
    for n, bits in [(1_000_000, 24), (37_001, 9)]:
        keys = rng.integers(0, 2 ** bits, n, dtype=np.uint64).astype(np.uint32)
        vals = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        want_k, want_v = _sort_allocating(engine, keys, vals, bits)
        got_k, got_v = _sort_noalloc(hrlib, keys, vals, bits)
        assert np.array_equal(got_k, want_k)
        assert np.array_equal(got_v, want_v)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(got_k, keys[order]) and np.array_equal(got_v, vals[order])


def test_noalloc_sort_rejects_sizes_beyond_its_scratch(hrlib):
    import torch
    n = (1 << 20) + 1
    tk = torch.zeros(n, dtype=torch.int32, device="cuda")
    tv = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = hrlib.hr_radix_sort_pairs_noalloc(None, C.c_void_p(tk.data_ptr()), C.c_void_p(tv.data_ptr()), n, 16)
    assert st == 1   # HR_ERR_INVALID_ARG
