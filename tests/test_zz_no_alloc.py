"""The allocation-free broad phase against the allocating one.

bgpu_broadphase_pairs_noalloc serves callers that cannot allocate device
memory while they run (a fixed device-memory budget, an allocator owned by
another runtime, a deadline that a cudaMalloc / cudaFree round trip would
break): they hand it device buffers and it keeps all of its scratch in one
fixed device array inside the library. This test calls it through the C ABI
on device buffers owned by the caller (torch tensors here) and checks that two
calls in a row return exactly the pairs of bgpu_broadphase_pairs, then that
inputs beyond its stated maximum are rejected. The file is collected last so a
run that stops at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from test_oracle_kats import ref_scattered_boxes

pytestmark = pytest.mark.gpu

BGPU_ERR_CAPACITY = 2


def _entry(bgpu_mod):
    f = bgpu_mod.lib().bgpu_broadphase_pairs_noalloc
    f.restype = ctypes.c_int32
    f.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64,
                  ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p]
    return f


def _inputs():
    big = np.array([[-1e30, -1e30, -1e30, 1e30, 1e30, 1e30]], dtype=np.float32)
    first = ref_scattered_boxes(0x5EED0001, 3000, 400, 300)
    first = np.concatenate([first[:1000], big, first[1000:], big], axis=0)  # two unbounded proxies
    second = ref_scattered_boxes(0x5EED0002, 700, 150, 200)  # smaller: stale scratch must not leak in
    return [first, second]


def test_noalloc_broadphase_matches_the_allocating_entry_point(gpu):
    import torch

    entry = _entry(gpu)
    for aabbs in _inputs():
        expected = gpu.broadphase_pairs(aabbs)
        a_dev = torch.from_numpy(np.ascontiguousarray(aabbs, dtype=np.float32)).cuda()
        cap = len(expected) + 32
        out = torch.full((cap, 2), -1, dtype=torch.int32, device="cuda")
        n_out = ctypes.c_uint64(0)
        torch.cuda.synchronize()
        status = entry(a_dev.data_ptr(), len(aabbs), out.data_ptr(), cap, ctypes.byref(n_out), None)
        torch.cuda.synchronize()
        assert status == 0, gpu.last_error()
        assert n_out.value == len(expected)
        got = out[: n_out.value].cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, expected)


def test_noalloc_broadphase_rejects_sizes_beyond_its_limits(gpu):
    import torch

    entry = _entry(gpu)
    n_out = ctypes.c_uint64(0)
    too_many = 65536 + 1
    a_dev = torch.zeros((too_many, 6), dtype=torch.float32, device="cuda")
    out = torch.zeros((16, 2), dtype=torch.int32, device="cuda")
    assert entry(a_dev.data_ptr(), too_many, out.data_ptr(), 16, ctypes.byref(n_out), None) == BGPU_ERR_CAPACITY
    assert "65536" in gpu.last_error()
    # Output buffer too small: the count comes back with BGPU_ERR_CAPACITY.
    aabbs = _inputs()[1]
    expected = gpu.broadphase_pairs(aabbs)
    a_small = torch.from_numpy(np.ascontiguousarray(aabbs, dtype=np.float32)).cuda()
    torch.cuda.synchronize()
    assert entry(a_small.data_ptr(), len(aabbs), out.data_ptr(), 16, ctypes.byref(n_out), None) == BGPU_ERR_CAPACITY
    assert n_out.value == len(expected)
