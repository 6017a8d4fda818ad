"""The tracer's radix sort (ptir_b200/csrc/radix_sort.cuh), which orders the LBVH's 60-bit Morton
keys and the wavefront's 28-bit ray-order keys, against numpy's stable sort: keys and values
equal, ties kept in input order. Sizes around the warp tile (2048 items) and the scan tile
(4096 counts), many duplicates and keys with bits outside the sorted range (which must not
count)."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "libptir_kat.so")


def _sort(keys: np.ndarray, vals: np.ndarray, begin: int, end: int):
    lib = C.CDLL(LIB)
    lib.ptirkat_radix_sort.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int,
                                       C.c_int]
    ki = torch.from_numpy(keys.view(np.int64 if keys.dtype == np.uint64 else np.int32).copy()).cuda()
    vi = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    ko, vo = torch.empty_like(ki), torch.empty_like(vi)
    rc = lib.ptirkat_radix_sort(keys.dtype.itemsize, ki.data_ptr(), ko.data_ptr(), vi.data_ptr(), vo.data_ptr(),
                                len(keys), begin, end)
    assert rc == 0
    return ko.cpu().numpy().view(keys.dtype), vo.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 31, 2047, 2048, 2049, 4096 * 3 + 5, 100_003, 1_048_579])
@pytest.mark.parametrize("dtype,begin,end", [(np.uint32, 0, 28), (np.uint64, 0, 60), (np.uint32, 4, 20)])
def test_radix_sort_matches_a_stable_sort(cuda_device, n, dtype, begin, end):
    rng = np.random.default_rng(n + end)
    bits = 8 * np.dtype(dtype).itemsize
    keys = rng.integers(0, np.iinfo(dtype).max, n, dtype=dtype, endpoint=True)
    # duplicates: a third of the keys repeat a few values in the sorted range
    dup = rng.random(n) < 0.33
    keys[dup] = (rng.integers(0, 7, int(dup.sum())).astype(dtype) << dtype(begin))
    vals = np.arange(n, dtype=np.uint32)
    ko, vo = _sort(keys, vals, begin, end)
    field = (keys >> dtype(begin)) & dtype((1 << (end - begin)) - 1) if end - begin < bits else keys >> dtype(begin)
    order = np.argsort(field, kind="stable")
    assert np.array_equal(vo, vals[order])
    assert np.array_equal(ko, keys[order])
