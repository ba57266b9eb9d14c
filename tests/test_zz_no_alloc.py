"""The allocation-free exclusive scan (lab_exclusive_scan_i64_noalloc).

It exists for callers that cannot allocate device memory when they call: a
process whose framework allocator already holds nearly all of the device, a host
thread that cannot wait on the driver's allocator, a deployment with a fixed
memory budget after start-up.  Its scratch is therefore a fixed array inside the
library.  This file sorts last so a run that stops at the first failure has run
everything else first; it must pass on its own in a fresh process and after the
other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from linalglib_b200 import _lib as L

pytestmark = pytest.mark.gpu

MAX_N = 65536 * 2048  # the documented limit: 134,217,728 elements


def _scan(gpu, fn, a):
    t = torch.as_tensor(a, dtype=torch.int64, device="cuda").clone()
    L.call(fn, t.numel(), gpu.ptr(t), gpu.stream_handle())
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _exclusive(a):
    out = np.zeros_like(a)
    np.cumsum(a[:-1], out=out[1:])
    return out


@pytest.mark.parametrize("sizes", [(5_000_011, 1_000_003), (1, 2), (2047, 2049),
                                   (2048, 4096), (4095, 6143), (6145, 2048 * 37 + 1)])
def test_noalloc_scan_matches_allocating_scan_twice(gpu, sizes):
    rng = np.random.default_rng(2024 + sizes[0])
    # two calls in a row on different data: the shared scratch keeps the first
    # call's contents, which must not leak into the second result
    for n in sizes:
        a = rng.integers(-7, 9, size=n)
        ref = _scan(gpu, "lab_exclusive_scan_i64", a)
        out = _scan(gpu, "lab_exclusive_scan_i64_noalloc", a)
        assert np.array_equal(out, ref)
        assert np.array_equal(out, _exclusive(a))


def test_noalloc_scan_at_its_size_limit(gpu):
    """n = 134,217,728, the largest size the fixed scratch covers (1 GiB of int64)."""
    rng = np.random.default_rng(7)
    a = rng.integers(-3, 4, size=MAX_N, dtype=np.int64)
    out = _scan(gpu, "lab_exclusive_scan_i64_noalloc", a)
    assert np.array_equal(out, _exclusive(a))


def test_noalloc_scan_rejects_sizes_beyond_its_scratch(gpu):
    t = torch.arange(16, dtype=torch.int64, device="cuda")
    before = t.clone()
    st = L.lib().lab_exclusive_scan_i64_noalloc(MAX_N + 1, C.c_void_p(t.data_ptr()),
                                                gpu.stream_handle())
    assert st == L.LAB_BAD_ARG
    assert "scratch" in L.lib().lab_last_error().decode()
    torch.cuda.synchronize()
    assert torch.equal(t, before)
