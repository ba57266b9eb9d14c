"""The allocation-free exclusive scan (lab_exclusive_scan_i64_noalloc).

It exists for callers that may not allocate device memory when they call
(graph recording without allocation nodes, threads that cannot wait on the
allocator, processes whose memory is fully reserved by another allocator), so
its scratch is a fixed array inside the library.  This file sorts last so a run
that stops at the first failure has run everything else first; it must pass on
its own in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from linalglib_b200 import _lib as L

pytestmark = pytest.mark.gpu

MAX_N = 65536 * 2048


def _scan(gpu, fn, a):
    t = torch.as_tensor(a, dtype=torch.int64, device="cuda").clone()
    L.call(fn, t.numel(), gpu.ptr(t), gpu.stream_handle())
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_noalloc_scan_matches_allocating_scan_twice(gpu):
    rng = np.random.default_rng(2024)
    # two calls in a row on different data: the shared scratch keeps the first
    # call's contents, which must not leak into the second result
    for n in (5_000_011, 1_000_003):
        a = rng.integers(-7, 9, size=n)
        ref = _scan(gpu, "lab_exclusive_scan_i64", a)
        out = _scan(gpu, "lab_exclusive_scan_i64_noalloc", a)
        assert np.array_equal(out, ref)
        assert out[0] == 0 and out[-1] == int(a[:-1].sum())


def test_noalloc_scan_rejects_sizes_beyond_its_scratch(gpu):
    t = torch.arange(16, dtype=torch.int64, device="cuda")
    before = t.clone()
    st = L.lib().lab_exclusive_scan_i64_noalloc(MAX_N + 1, C.c_void_p(t.data_ptr()),
                                                gpu.stream_handle())
    assert st == L.LAB_BAD_ARG
    assert "scratch" in L.lib().lab_last_error().decode()
    torch.cuda.synchronize()
    assert torch.equal(t, before)
