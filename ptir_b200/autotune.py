"""Launch-shape autotuner of the wavefront tracer.

Sweeps the k-buffer size (8, 16, 32), the block size (64, 128, 256), the chunk size (tiles of 8x4
paths per chunk) and the intersection refill threshold, timing each candidate with CUDA events
on a caller-supplied sample of the workload (one forward + adjoint, after a warm-up call), and
returns the fastest. Results are cached per GPU and workload signature in a JSON file.

A k-buffer size other than the reference's 16 moves the distance at which subtrees are culled.
That changes which grazing candidates (closest approach before their own box entry) are found,
and some of them are accepted, so the image changes. On the 300k-Gaussian config-4 scene, K 32
changes 0.3 % of samples, some by more than 1 in HDR. Pass ``kbuffers=(16,)`` to tune only
shapes whose results are the reference's.
"""
from __future__ import annotations

import itertools
import json
import os
from dataclasses import asdict, dataclass
from typing import Callable, Iterable

import torch

KBUFFERS = (8, 16, 32)
BLOCKS = (64, 128, 256)
CHUNKS = (0, 131072)  # 0: the tracer sizes its chunk from the free device memory
REFILLS = (16, 32)


@dataclass(frozen=True)
class Shape:
    kbuffer: int = 16
    block_size: int = 128
    chunk_tiles: int = 0
    refill_lanes: int = 32

    def launch(self) -> dict:
        """Keyword arguments of OptixTracer for this shape."""
        return asdict(self)


def space(kbuffers: Iterable[int] = KBUFFERS, blocks: Iterable[int] = BLOCKS, chunks: Iterable[int] = CHUNKS,
          refills: Iterable[int] = REFILLS) -> list:
    return [Shape(k, b, c, r) for k, b, c, r in itertools.product(kbuffers, blocks, chunks, refills)]


def pick(timings: dict) -> Shape:
    """The fastest shape of {Shape: milliseconds}; ties go to the reference's k-buffer size, then
    to the smaller block and chunk (the order of the sweep)."""
    if not timings:
        raise ValueError("no timings")
    return min(timings, key=lambda s: (timings[s], s.kbuffer != 16, s.block_size, s.chunk_tiles, s.refill_lanes))


def time_shape(make_tracer: Callable[..., object], run: Callable[[object], None], shape: Shape, repeats: int = 2) -> float:
    """Median milliseconds of run(tracer) for a tracer built with the shape (one warm-up call)."""
    tr = make_tracer(**shape.launch())
    run(tr)
    torch.cuda.synchronize()
    times = []
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        run(tr)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    del tr
    times.sort()
    return times[len(times) // 2]


class Autotuner:
    """Sweep-and-cache tuner: ``tune(signature, make_tracer, run)`` returns the best Shape for the
    signature (a string naming the workload: Gaussian count, samples, bounces, storage, ...)."""

    def __init__(self, cache_path: str | None = None):
        self.cache_path = cache_path
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    @staticmethod
    def _key(signature: str) -> str:
        dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
        return f"{dev}|{signature}"

    def tune(self, signature: str, make_tracer: Callable[..., object], run: Callable[[object], None],
             shapes: list | None = None, repeats: int = 2) -> tuple:
        """(best Shape, {shape: ms}) — from the cache when the signature was tuned on this GPU."""
        key = self._key(signature)
        if key in self.cache:
            entry = self.cache[key]
            return Shape(**entry["best"]), {}
        timings = {s: time_shape(make_tracer, run, s, repeats) for s in (shapes or space())}
        best = pick(timings)
        self.cache[key] = {"best": asdict(best),
                           "timings_ms": [dict(asdict(s), ms=round(ms, 3)) for s, ms in timings.items()]}
        if self.cache_path:
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1)
            os.replace(tmp, self.cache_path)
        return best, timings
