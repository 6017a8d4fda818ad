"""Autotuner logic without a GPU: the pick rule, the search space and the cache."""
import json

import pytest

from ptir_b200 import autotune as A


def test_space_covers_the_benchmark_sweep():
    shapes = A.space()
    assert len(shapes) == len(A.KBUFFERS) * len(A.BLOCKS) * len(A.CHUNKS) * len(A.REFILLS)
    assert {s.kbuffer for s in shapes} == {8, 16, 32} and {s.block_size for s in shapes} == {64, 128, 256}


def test_pick_fastest_with_ties_to_reference_kbuffer():
    a, b, c = A.Shape(8, 64, 32768, 32), A.Shape(16, 128, 131072, 32), A.Shape(32, 256, 131072, 16)
    assert A.pick({a: 3.0, b: 2.0, c: 2.5}) == b
    assert A.pick({a: 2.0, b: 2.0}) == b  # tie: the reference's k-buffer size
    with pytest.raises(ValueError):
        A.pick({})


def test_cached_signature_skips_the_sweep(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setattr(A.Autotuner, "_key", staticmethod(lambda sig: "dev|" + sig))
    best = A.Shape(16, 64, 32768, 16)
    path.write_text(json.dumps({"dev|scene": {"best": best.launch(), "timings_ms": []}}))
    tuner = A.Autotuner(str(path))

    def boom(**kw):
        raise AssertionError("the sweep must not run for a cached signature")

    got, timings = tuner.tune("scene", boom, lambda tr: None)
    assert got == best and timings == {}
