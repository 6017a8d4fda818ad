"""The allocation-free scene-bounds entry point (ptir_instance_bounds_noalloc).

It serves callers that cannot allocate device memory once running: a process that reserves
all device memory for its own pool, or a plugin whose host forbids device allocation after
start-up. The test calls it through the C ABI and checks its result against the existing
path (ptir_build_bvh + ptir_scene_bounds) on two calls in a row, for each attribute storage
(FP32, and BF16 / FP16, where both round the attributes the same way). The second call covers
fewer Gaussians than the first, so stale scratch from the first call must not leak into it. An
empty scene gives the empty box. This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from ptir_b200 import _native
from tests.scenes import make_tracer, small_scene

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-7


def _bind():
    lib = _native.load()
    fn = lib.ptir_instance_bounds_noalloc
    fn.argtypes = [C.c_float, C.c_float, C.c_int32, C.c_int32] + [C.c_void_p] * 4 + [C.c_int32, C.c_void_p,
                                                                                     C.c_void_p, C.c_char_p, C.c_int32]
    fn.restype = C.c_int
    return fn


STORAGES = {"fp32": 0, "bf16": 1, "fp16": 2}


def _noalloc_bounds(fn, S, n, storage="fp32"):
    out = torch.full((8,), float("nan"), dtype=torch.float32, device="cuda")
    err = C.create_string_buffer(256)
    rc = fn(4.0, 0.0113, 1, STORAGES[storage], S["build_pos"].data_ptr(), S["build_rot"].data_ptr(),
            S["build_scl"].data_ptr(), S["build_dns"].data_ptr(), n, out.data_ptr(),
            torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return np.concatenate([o[0:3], o[4:7]])


@pytest.mark.parametrize("storage", ["fp32", "bf16", "fp16"])
def test_noalloc_bounds_match_build_bvh(cuda_device, storage):
    fn = _bind()
    tr = make_tracer(storage=storage)
    for n, seed in ((6000, 1), (1500, 2)):  # two calls in a row, the second one smaller
        s = small_scene(n=n, w=8, h=8, seed=seed, layout="cluster_shell", scale_range=(0.002, 0.2))
        S = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in s.items()
             if k.startswith("build_")}
        got = _noalloc_bounds(fn, S, n, storage)
        tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], True, True)
        ref = tr.scene_bounds().numpy()
        assert np.allclose(got, ref, rtol=RTOL, atol=ATOL), (storage, n, got, ref)


def test_noalloc_empty_scene_gives_the_empty_box(cuda_device):
    fn = _bind()
    S = {k: torch.zeros((1, c), dtype=torch.float32, device="cuda")
         for k, c in (("build_pos", 3), ("build_rot", 4), ("build_scl", 3), ("build_dns", 1))}
    got = _noalloc_bounds(fn, S, 0)
    assert np.all(got[:3] >= 1e38) and np.all(got[3:] <= -1e38), got


def test_noalloc_rejects_too_many_gaussians(cuda_device):
    fn = _bind()
    out = torch.empty((8,), dtype=torch.float32, device="cuda")
    err = C.create_string_buffer(256)
    rc = fn(4.0, 0.0113, 1, 0, None, None, None, None, 8_388_609, out.data_ptr(), None, err, 256)
    assert rc == _native.PTIR_EINVAL
    assert b"exceeds the allocation-free limit" in err.value
