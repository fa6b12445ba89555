"""The allocation-free scan entry point (gcmfgh_exclusive_scan_i32_noalloc).

It exists for callers that cannot let the library allocate device memory: engines that
keep every device byte under their own pool, or latency-sensitive loops that must not
trigger cudaMalloc's implicit synchronisation.  Its scratch is a fixed array inside the
library, so this test checks, through the C ABI, that two calls in a row (the second
reusing the array the first left behind) give exactly the output of the allocating
gcmfgh_exclusive_scan_i32, and that sizes beyond the fixed maximum are refused.
The file name sorts last so that a run stopping at the first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest

from conftest import build_library

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 1 << 24   # GCMFGH_NOALLOC_SCAN_MAX_ELEMENTS


def _lib():
    L = ctypes.CDLL(build_library())
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    L.gcmfgh_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.gcmfgh_destroy.argtypes = [vp]
    L.gcmfgh_exclusive_scan_i32.argtypes = [vp, vp, vp, i64, ctypes.POINTER(i64)]
    L.gcmfgh_exclusive_scan_i32_noalloc.argtypes = [vp, vp, i64, vp, vp]
    return L


def test_noalloc_scan_equals_allocating_scan_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _lib()
    ctx = ctypes.c_void_p()
    assert L.gcmfgh_create(0, ctypes.byref(ctx)) == 0
    try:
        rng = np.random.default_rng(1234)
        # two calls in a row; the second is smaller, so stale status words of the first
        # call would corrupt it if the scratch were not cleared
        # the third call is all negative, so every tile aggregate and running prefix
        # that the look-back passes between tiles is negative
        for n, lo, hi in ((3_000_017, -1000, 100000), (1_234_567, -1000, 100000), (3_000_017, -1000, 0)):
            a = torch.from_numpy(rng.integers(lo, hi, size=n).astype(np.int32)).cuda()
            ref = torch.empty(n, dtype=torch.int64, device="cuda")
            ref_total = ctypes.c_int64()
            assert L.gcmfgh_exclusive_scan_i32(ctx, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                               n, ctypes.byref(ref_total)) == 0
            out = torch.full((n,), -7, dtype=torch.int64, device="cuda")
            total = torch.full((1,), -7, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            st = L.gcmfgh_exclusive_scan_i32_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                     n, ctypes.c_void_p(total.data_ptr()), None)
            assert st == 0
            assert torch.equal(out, ref)
            assert int(total.item()) == ref_total.value
            expect = np.concatenate([[0], np.cumsum(a.cpu().numpy(), dtype=np.int64)])
            assert np.array_equal(out.cpu().numpy(), expect[:-1]) and ref_total.value == int(expect[-1])
    finally:
        L.gcmfgh_destroy(ctx)


def test_noalloc_scan_refuses_sizes_beyond_its_maximum():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _lib()
    dummy = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = L.gcmfgh_exclusive_scan_i32_noalloc(ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()),
                                             MAX_ELEMENTS + 1, None, None)
    assert st == 1   # GCMFGH_INVALID_ARGUMENT, before any GPU work
