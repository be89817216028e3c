"""Device radix sort: keys bit-exact against the oracle's restatement of the reference
key (particle_sort.wgsl:94-102) and a Python tile key; permutation equal to a stable
argsort (ties in input order)."""
import ctypes

import numpy as np
import pytest

from oracle.oracle import lib as oracle_lib

pytestmark = pytest.mark.gpu


def tile_key(xy, res):
    cx = np.clip(np.floor(xy[:, 0]), 0, res - 1).astype(np.uint32)
    cy = np.clip(np.floor(xy[:, 1]), 0, res - 1).astype(np.uint32)
    tx, ty = cx >> 3, cy >> 3
    m = np.zeros_like(tx)
    for b in range(16):
        m |= ((tx >> b) & 1) << (2 * b) | ((ty >> b) & 1) << (2 * b + 1)
    return (m << 6) | ((cx & 7) << 3) | (cy & 7)


def device_sort(cuda_lib, xy, res, mode):
    n = len(xy)
    xy = np.ascontiguousarray(xy, dtype=np.float32)
    keys = np.zeros(n, dtype=np.uint32)
    perm = np.zeros(n, dtype=np.uint32)
    st = cuda_lib.emerge_cuda_sort_keys(xy.ctypes.data_as(ctypes.c_void_p), n, res, mode,
                                        keys.ctypes.data_as(ctypes.c_void_p),
                                        perm.ctypes.data_as(ctypes.c_void_p))
    assert st == 0
    return keys, perm


@pytest.mark.parametrize("n,res", [(1, 64), (1000, 64), (70_001, 512), (1_000_003, 1024)])
def test_block_index_keys_and_stable_perm(cuda_lib, n, res):
    rng = np.random.default_rng(n)
    xy = rng.uniform(-3.0, res + 3.0, size=(n, 2)).astype(np.float32)
    xy[: n // 10] = np.floor(xy[: n // 10])  # exact cell boundaries
    keys, perm = device_sort(cuda_lib, xy, res, 1)
    L = oracle_lib()
    ref = np.array([L.oracle_block_index(float(a), float(b), res) for a, b in xy[:2000]],
                   dtype=np.uint32)
    np.testing.assert_array_equal(keys[:2000], ref)
    np.testing.assert_array_equal(perm, np.argsort(keys, kind="stable").astype(np.uint32))


@pytest.mark.parametrize("n,res", [(5, 16), (4097, 128), (600_000, 1024), (2_000_000, 4096)])
def test_tile_keys_and_stable_perm(cuda_lib, n, res):
    rng = np.random.default_rng(n + res)
    xy = rng.uniform(0.0, res, size=(n, 2)).astype(np.float32)
    xy[::7] = xy[0]  # many ties
    keys, perm = device_sort(cuda_lib, xy, res, 0)
    np.testing.assert_array_equal(keys, tile_key(xy, res))
    np.testing.assert_array_equal(perm, np.argsort(keys, kind="stable").astype(np.uint32))
    # and the oracle's stable argsort agrees
    oref = np.zeros(n, dtype=np.uint32)
    oracle_lib().oracle_stable_argsort_u32(keys.ctypes.data_as(ctypes.c_void_p), n,
                                           oref.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_array_equal(perm, oref)
