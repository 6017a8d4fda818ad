"""The autotuner times real launch shapes on a small scene and returns one of them; the tuned
tracer renders what the default one does (shapes with the reference's k-buffer size change no
result)."""
import pytest
import torch

from ptir_b200 import autotune as A
from tests.scenes import gpu_trace, make_tracer, small_scene, to_torch

pytestmark = pytest.mark.gpu


def test_tune_small_scene(cuda_device, tmp_path):
    S = to_torch(small_scene(n=2000, w=48, h=40, spp=2, max_bounces=3))

    def run(tr):
        gpu_trace(tr, S)

    shapes = A.space(kbuffers=(16,), blocks=(64, 128), chunks=(8, 131072), refills=(32,))
    tuner = A.Autotuner(str(tmp_path / "tune.json"))
    best, timings = tuner.tune("small-scene", make_tracer, run, shapes=shapes, repeats=1)
    assert best in shapes and len(timings) == len(shapes) and all(t > 0 for t in timings.values())
    again, cached = A.Autotuner(str(tmp_path / "tune.json")).tune("small-scene", make_tracer, run, shapes=shapes)
    assert again == best and cached == {}
    a = [t.clone() for t in gpu_trace(make_tracer(), S)]
    b = gpu_trace(make_tracer(**best.launch()), S)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
