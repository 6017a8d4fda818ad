"""ptir_b200 — B200-native drop-in for PTIR's differentiable Gaussian-field path tracer.

``OptixTracer`` mirrors the reference's native object (trace / trace_bwd / build_bvh) on top of
``libptir_b200.so``; ``Tracer`` mirrors the Python ``threedgptir_tracer.Tracer`` above it.
"""
from .optix_tracer import OptixTracer  # noqa: F401

__all__ = ["OptixTracer", "Tracer", "LightBuffers"]


def __getattr__(name):
    if name in ("Tracer", "LightBuffers"):
        from . import tracer

        return getattr(tracer, name)
    raise AttributeError(name)
