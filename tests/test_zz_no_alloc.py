"""The allocation-free preprocessing entry point (pacmap_preprocess_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory themselves -- their device memory belongs to
another framework's allocator or to a fixed budget, or they run a latency-critical loop that must not
reach cudaMalloc/cudaFree. Its output must equal the allocating entry point's (pacmap_preprocess)
bit for bit, call after call, although both calls share one fixed scratch array.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_D = 16384  # the scratch array's stated limit


def _entry(lib):
    fn = lib._abi.lib().pacmap_preprocess_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int32]
    return fn


def test_noalloc_preprocess_matches_allocating_entry_point(lib):
    import torch

    fn = _entry(lib)
    stream = torch.cuda.current_stream()
    # Two calls in a row with different data and shapes: the second must not see the first's scratch.
    for seed, (n, d), (lo, hi) in [(11, (5000, 37), (-3.0, 5.0)), (12, (3001, 128), (2.0, 9.0))]:
        x = np.random.default_rng(seed).uniform(lo, hi, size=(n, d)).astype(np.float32)
        expected, *_ = lib.stages.preprocess(x)
        dx = torch.from_numpy(x).cuda()
        dout = torch.empty_like(dx)
        rc = fn(C.c_void_p(dx.data_ptr()), n, d, C.c_void_p(dout.data_ptr()), C.c_void_p(stream.cuda_stream), 0)
        stream.synchronize()
        assert rc == 0, lib._abi.last_error()
        got = dout.cpu().numpy()
        # same arithmetic as the allocating entry point: exact equality is the tolerance
        assert np.array_equal(got, expected)


def test_noalloc_in_place_small_n_keeps_device_and_memory(lib):
    import torch

    fn = _entry(lib)
    stream = torch.cuda.current_stream()
    # n < 512 (one column-sum chunk), and the output written over the input
    x = np.random.default_rng(13).uniform(-1.0, 4.0, size=(300, 65)).astype(np.float32)
    expected, *_ = lib.stages.preprocess(x)
    dx = torch.from_numpy(x).cuda()
    rc = fn(C.c_void_p(dx.data_ptr()), 300, 65, C.c_void_p(dx.data_ptr()), C.c_void_p(stream.cuda_stream), 0)
    stream.synchronize()
    assert rc == 0, lib._abi.last_error()
    assert np.array_equal(dx.cpu().numpy(), expected)
    # later calls take no device memory: free memory is unchanged across two more calls
    y = torch.from_numpy(np.random.default_rng(14).normal(size=(2000, 48)).astype(np.float32)).cuda()
    out = torch.empty_like(y)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert fn(C.c_void_p(y.data_ptr()), 2000, 48, C.c_void_p(out.data_ptr()), None, 0) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    # the caller's current device is left as it was
    assert torch.cuda.current_device() == 0


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    import torch

    fn = _entry(lib)
    d = MAX_D + 1
    dx = torch.zeros((2, d), dtype=torch.float32, device="cuda")
    dout = torch.empty_like(dx)
    rc = fn(C.c_void_p(dx.data_ptr()), 2, d, C.c_void_p(dout.data_ptr()), None, 0)
    assert rc == lib.Unsupported.code
    assert "16384" in lib._abi.last_error()
