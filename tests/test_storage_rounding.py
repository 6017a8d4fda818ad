"""The numpy rounding that models the tracer's 16-bit attribute storage matches torch's
float32 -> bfloat16 / float16 conversion (round to nearest even) on random and edge values."""
import numpy as np
import pytest
import torch

from tests.scenes import round_to


@pytest.mark.parametrize("storage,dtype", [("bf16", torch.bfloat16), ("fp16", torch.float16)])
def test_round_to_matches_torch(storage, dtype):
    rng = np.random.default_rng(0)
    a = np.concatenate([
        rng.standard_normal(100000).astype(np.float32) * np.float32(10.0) ** rng.integers(-6, 4, 100000),
        np.array([0.0, -0.0, 1.0, -1.0, 0.002, 0.2, 20.0, 1.00390625, 1.01171875, 65504.0, 3.0e-5], np.float32),
    ]).astype(np.float32)
    want = torch.from_numpy(a).to(dtype).to(torch.float32).numpy()
    got = round_to(a, storage)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
