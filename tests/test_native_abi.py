"""The C-ABI library loads and exports every entry point declared in include/ptir_b200.h."""
import ctypes
import os
import re

from ptir_b200 import _native, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "ptir_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(ptir_[a-z_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    path = build.build()
    lib = ctypes.CDLL(path)
    names = _declared()
    assert "ptir_trace" in names and "ptir_trace_bwd" in names and "ptir_build_bvh" in names
    for name in names:
        assert hasattr(lib, name), name
    assert set(_native.EXPORTS) <= set(names)


def test_abi_version_without_gpu():
    lib = _native.load()
    assert lib.ptir_abi_version() == _native.ABI_VERSION == 6


def test_built_for_sm100a():
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH_FLAGS)


def test_unknown_names_are_rejected_before_the_device():
    """A misspelt storage or hierarchy builder fails with a clear ValueError before any device
    call (CPU only)."""
    import pytest

    from ptir_b200 import OptixTracer

    args = ("", "", "reference", "referenceBwd", "instances", 4, 0.0113, True, 3, True, True, True, False, False)
    with pytest.raises(ValueError, match="bvh_builder"):
        OptixTracer(*args, bvh_builder="sah")
    with pytest.raises(ValueError, match="storage"):
        OptixTracer(*args, storage="fp8")
