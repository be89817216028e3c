"""Allocation-free sort entry point (emerge_cuda_sort_keys_noalloc), for callers that cannot
let a library allocate: cudaMalloc/cudaFree synchronise the whole device, and a caller whose
memory pool holds the device's memory would see them fail.  With caller-owned device buffers
and the caller's stream it returns the same keys and stable permutation as the allocating
emerge_cuda_sort_keys, and the device's free memory does not change across its calls.  Named
to be collected last, so it runs both alone and after every other test in the same process."""
import ctypes

import numpy as np
import pytest

from emerge_engine_b200 import abi

MAX = 65536  # EMERGE_SORT_NOALLOC_MAX


def allocating_sort(cuda_lib, xy, res, mode):
    n = len(xy)
    keys = np.zeros(n, dtype=np.uint32)
    perm = np.zeros(n, dtype=np.uint32)
    st = cuda_lib.emerge_cuda_sort_keys(xy.ctypes.data_as(ctypes.c_void_p), n, res, mode,
                                        keys.ctypes.data_as(ctypes.c_void_p),
                                        perm.ctypes.data_as(ctypes.c_void_p))
    assert st == 0, cuda_lib.emerge_cuda_last_global_error()
    return keys, perm


def test_rejects_more_than_the_maximum_before_device_work(cuda_lib):
    """Runs without a GPU too: the size check precedes every CUDA call."""
    p = ctypes.c_void_p(256)
    st = cuda_lib.emerge_cuda_sort_keys_noalloc(p, MAX + 1, 64, 0, p, p, None)
    assert st == abi.ERR_INVALID_ARG
    assert b"EMERGE_SORT_NOALLOC_MAX" in cuda_lib.emerge_cuda_last_global_error()
    assert cuda_lib.emerge_cuda_sort_keys_noalloc(p, 16, 64, 2, p, p, None) == abi.ERR_INVALID_ARG


@pytest.mark.parametrize("res", [0, 32769, 1 << 20])
def test_rejects_grid_res_outside_the_range_before_device_work(cuda_lib, res):
    """grid_res must lie in 1..32768; checked before any CUDA call (runs without a GPU)."""
    p = ctypes.c_void_p(256)
    assert cuda_lib.emerge_cuda_sort_keys_noalloc(p, 16, res, 0, p, p, None) == abi.ERR_INVALID_ARG
    assert b"grid_res in 1..32768" in cuda_lib.emerge_cuda_last_global_error()


def _noalloc_sort(cuda_lib, n, res, mode, d_xy, d_keys, d_perm, stream):
    st = cuda_lib.emerge_cuda_sort_keys_noalloc(
        ctypes.c_void_p(d_xy.data_ptr()), n, res, mode, ctypes.c_void_p(d_keys.data_ptr()),
        ctypes.c_void_p(d_perm.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert st == 0, cuda_lib.emerge_cuda_last_global_error()


@pytest.mark.gpu
@pytest.mark.parametrize("mode,res", [(0, 1024), (1, 256), (0, 32768), (1, 32768)])
def test_matches_the_allocating_sort_two_calls_in_a_row(cuda_lib, mode, res):
    import torch

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(1234 + mode + res)
    cases = []
    for n in (MAX, 40_001):  # the second call is smaller: nothing of the first may leak
        xy = rng.uniform(-2.0, res + 2.0, size=(n, 2)).astype(np.float32)
        xy[::5] = xy[3]  # many equal keys: the permutation must keep input order
        xy[: n // 8] = np.floor(xy[: n // 8])  # exact cell boundaries
        keys, perm = allocating_sort(cuda_lib, xy, res, mode)
        d_xy = torch.from_numpy(xy).to(dev)
        d_keys = torch.full((n,), -1, dtype=torch.int32, device=dev)
        d_perm = torch.full((n,), -1, dtype=torch.int32, device=dev)
        cases.append((n, keys, perm, d_xy, d_keys, d_perm))
    side = torch.cuda.Stream(dev)
    # Warm-up call on buffers of its own: the first call on a device may load this part of
    # the library's device image, which is when the driver reserves the fixed working array.
    w_xy = torch.zeros((64, 2), dtype=torch.float32, device=dev)
    w_keys = torch.zeros(64, dtype=torch.int32, device=dev)
    w_perm = torch.zeros(64, dtype=torch.int32, device=dev)
    _noalloc_sort(cuda_lib, 64, res, mode, w_xy, w_keys, w_perm, side)
    side.synchronize()
    torch.cuda.synchronize(dev)
    free_before = torch.cuda.mem_get_info(dev)[0]

    for n, _, _, d_xy, d_keys, d_perm in cases:  # both calls queued back to back
        _noalloc_sort(cuda_lib, n, res, mode, d_xy, d_keys, d_perm, side)
    side.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free_before, "device memory was allocated"

    for n, keys, perm, _, d_keys, d_perm in cases:
        np.testing.assert_array_equal(d_keys.cpu().numpy().view(np.uint32), keys)
        np.testing.assert_array_equal(d_perm.cpu().numpy().view(np.uint32), perm)
        np.testing.assert_array_equal(perm, np.argsort(keys, kind="stable").astype(np.uint32))


@pytest.mark.gpu
def test_rejects_host_memory(cuda_lib):
    import torch

    torch.cuda.init()
    xy = np.zeros((8, 2), dtype=np.float32)
    out = np.zeros(8, dtype=np.uint32)
    st = cuda_lib.emerge_cuda_sort_keys_noalloc(
        xy.ctypes.data_as(ctypes.c_void_p), 8, 64, 0, out.ctypes.data_as(ctypes.c_void_p),
        out.ctypes.data_as(ctypes.c_void_p), None)
    assert st == abi.ERR_INVALID_ARG
