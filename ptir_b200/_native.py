"""ctypes binding of ``libptir_b200.so`` (the C ABI declared in include/ptir_b200.h).

The library is the only compute path: if it cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

_LIB = None

ABI_VERSION = 6  # PTIR_ABI_VERSION of include/ptir_b200.h that these structs mirror
PTIR_OK = 0
PTIR_EINVAL = 1
PTIR_ECUDA = 2
PTIR_ESTATE = 3
PTIR_EDEVICE = 4

_FP = C.c_void_p  # device pointers are passed as integers


class PtirConfig(C.Structure):
    _fields_ = [
        ("kernel_degree", C.c_float),
        ("kernel_min_response", C.c_float),
        ("density_clamping", C.c_int32),
        ("sph_degree", C.c_int32),
        ("enable_normals", C.c_int32),
        ("enable_hitcounts", C.c_int32),
        ("enable_mis", C.c_int32),
        ("enable_metallic", C.c_int32),
        ("visualize_lights", C.c_int32),
        ("collect_counters", C.c_int32),
        ("schedule", C.c_int32),
        ("chunk_tiles", C.c_int32),
        ("kbuffer", C.c_int32),
        ("refill_lanes", C.c_int32),
        ("block_size", C.c_int32),
        ("collect_timings", C.c_int32),
        ("ray_order", C.c_int32),
        ("exact_replay", C.c_int32),
        ("grad_sums", C.c_int32),
        ("storage", C.c_int32),
        ("grad_aggregate", C.c_int32),
        ("shadow_kbuffer", C.c_int32),
        ("exact_candidates", C.c_int32),
        ("resume_rounds", C.c_int32),
        ("bvh_builder", C.c_int32),
    ]


STORAGES = {"fp32": 0, "bf16": 1, "fp16": 2}
BVH_BUILDERS = {"default": 0, "morton": 1, "ploc": 2}
STAGES = ("intersect", "shadow", "replay", "shading", "megakernel", "sort")


class PtirView(C.Structure):
    _fields_ = [("z", C.c_int32), ("h", C.c_int32), ("w", C.c_int32), ("frame", C.c_uint32), ("ray_to_world", _FP)]


MAX_VIEWS = 64


class PtirStageTimes(C.Structure):
    _fields_ = [("ms", C.c_double * len(STAGES)), ("launches", C.c_uint64 * len(STAGES))]


SCHEDULES = {"wavefront": 0, "megakernel": 1}


class PtirTraceArgs(C.Structure):
    _fields_ = [
        ("frame", C.c_uint32),
        ("ray_to_world", _FP),
        ("ray_origin", _FP),
        ("ray_direction", _FP),
        ("z", C.c_int32), ("h", C.c_int32), ("w", C.c_int32),
        ("particle_density", _FP),
        ("particle_material", _FP),
        ("particle_radiance", _FP),
        ("particle_shading_normal", _FP),
        ("n", C.c_int32),
        ("environment", _FP),
        ("env_h", C.c_int32), ("env_w", C.c_int32),
        ("environment_alias", _FP),
        ("alias_h", C.c_int32), ("alias_w", C.c_int32),
        ("lights", _FP), ("light_alias", _FP), ("mesh_light_vertices", _FP),
        ("mesh_light_triangles", _FP), ("mesh_lights", _FP), ("mesh_light_alias", _FP),
        ("num_lights", C.c_int32), ("num_light_entries", C.c_int32), ("num_mesh_lights", C.c_int32),
        ("num_mesh_light_vertices", C.c_int32), ("num_mesh_light_triangles", C.c_int32),
        ("mesh_light_alias_cols", C.c_int32),
        ("sh_indirect", C.c_uint32),
        ("sph_eval_degree", C.c_int32),
        ("min_transmittance", C.c_float),
        ("max_bounces", C.c_uint32),
        ("use_strides", C.c_int32),
        ("ray_origin_strides", C.c_int64 * 4),
        ("ray_direction_strides", C.c_int64 * 4),
    ]


class PtirTraceOutputs(C.Structure):
    _fields_ = [(k, _FP) for k in (
        "radiance", "density", "hit_distance", "hit_distance_second_moment", "depth_distortion", "normal",
        "shading_normal", "material", "hits_count", "pbr", "light", "pbr_components", "visibility",
        "path_signature")]


class PtirBwdArgs(C.Structure):
    _fields_ = [(k, _FP) for k in ("pbr", "light", "pbr_grad", "light_grad", "material_grad")] + [
        ("use_strides", C.c_int32)] + [
        (k + "_strides", C.c_int64 * 4) for k in ("pbr", "light", "pbr_grad", "light_grad", "material_grad")]


class PtirBwdOutputs(C.Structure):
    _fields_ = [("particle_material_grad", _FP), ("environment_grad", _FP)]


class PtirCounters(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("segments", "trace_calls", "candidates", "accepted", "env_lookups", "replay",
                                          "replay_accepted", "node_visits", "leaf_tests")]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


EXPORTS = ("ptir_abi_version", "ptir_create", "ptir_destroy", "ptir_build_bvh", "ptir_trace", "ptir_trace_bwd",
           "ptir_trace_views", "ptir_trace_bwd_views", "ptir_get_counters", "ptir_get_stage_counters", "ptir_get_stage_times", "ptir_set_collect_timings", "ptir_device_status",
           "ptir_scene_bounds", "ptir_debug_accel", "ptir_selective_adam", "ptir_env_table_scratch_bytes",
           "ptir_build_env_table", "ptir_last_error")


def lib_path() -> str:
    """The library loaded: $PTIR_B200_LIBRARY when set (a build kept elsewhere, loaded as it is),
    else the in-tree build."""
    return os.environ.get("PTIR_B200_LIBRARY") or _build.LIB_PATH


def load(build_if_missing: bool = True):
    """Load the shared library (building the in-tree one first when it is missing or stale)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if build_if_missing and not os.environ.get("PTIR_B200_LIBRARY") and _build.needs_build():
        _build.build()
    path = lib_path()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: run `python -m ptir_b200.build`")
    L = C.CDLL(path)
    P = C.POINTER
    L.ptir_abi_version.restype = C.c_int
    if L.ptir_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{path} has ABI version {L.ptir_abi_version()}, these bindings need {ABI_VERSION}: "
                           "rebuild it (python -m ptir_b200.build)")
    L.ptir_create.argtypes = [P(PtirConfig), P(C.c_void_p)]
    L.ptir_create.restype = C.c_int
    L.ptir_destroy.argtypes = [C.c_void_p]
    L.ptir_destroy.restype = None
    L.ptir_build_bvh.argtypes = [C.c_void_p, _FP, _FP, _FP, _FP, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    L.ptir_build_bvh.restype = C.c_int
    L.ptir_trace.argtypes = [C.c_void_p, P(PtirTraceArgs), P(PtirTraceOutputs), C.c_void_p]
    L.ptir_trace.restype = C.c_int
    L.ptir_trace_bwd.argtypes = [C.c_void_p, P(PtirTraceArgs), P(PtirBwdArgs), P(PtirBwdOutputs), C.c_void_p]
    L.ptir_trace_bwd.restype = C.c_int
    L.ptir_trace_views.argtypes = [C.c_void_p, P(PtirTraceArgs), P(PtirView), C.c_int32, P(PtirTraceOutputs),
                                   C.c_void_p]
    L.ptir_trace_views.restype = C.c_int
    L.ptir_trace_bwd_views.argtypes = [C.c_void_p, P(PtirTraceArgs), P(PtirView), C.c_int32, P(PtirBwdArgs),
                                       P(PtirBwdOutputs), C.c_void_p]
    L.ptir_trace_bwd_views.restype = C.c_int
    L.ptir_get_counters.argtypes = [C.c_void_p, P(PtirCounters), C.c_void_p]
    L.ptir_get_counters.restype = C.c_int
    L.ptir_get_stage_counters.argtypes = [C.c_void_p, C.c_int32, P(PtirCounters), C.c_void_p]
    L.ptir_get_stage_counters.restype = C.c_int
    L.ptir_get_stage_times.argtypes = [C.c_void_p, P(PtirStageTimes)]
    L.ptir_get_stage_times.restype = C.c_int
    L.ptir_set_collect_timings.argtypes = [C.c_void_p, C.c_int32]
    L.ptir_set_collect_timings.restype = C.c_int
    L.ptir_device_status.argtypes = [C.c_void_p, P(C.c_uint32), C.c_void_p]
    L.ptir_device_status.restype = C.c_int
    L.ptir_scene_bounds.argtypes = [C.c_void_p, P(C.c_float), C.c_void_p]
    L.ptir_scene_bounds.restype = C.c_int
    L.ptir_debug_accel.argtypes = [C.c_void_p, _FP, _FP, C.c_void_p]
    L.ptir_debug_accel.restype = C.c_int
    L.ptir_selective_adam.argtypes = [_FP, _FP, _FP, _FP, _FP, C.c_int64, C.c_int32, C.c_float, C.c_float, C.c_float,
                                      C.c_float, C.c_void_p]
    L.ptir_selective_adam.restype = C.c_int
    L.ptir_env_table_scratch_bytes.argtypes = [C.c_int32]
    L.ptir_env_table_scratch_bytes.restype = C.c_size_t
    L.ptir_build_env_table.argtypes = [_FP, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _FP, _FP,
                                       C.c_size_t, C.c_void_p]
    L.ptir_build_env_table.restype = C.c_int
    L.ptir_last_error.argtypes = [C.c_void_p]
    L.ptir_last_error.restype = C.c_char_p
    _LIB = L
    return L


class PtirError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"ptir error {code}: {message}")
        self.code = code


def check(handle, rc: int, what: str) -> None:
    if rc != PTIR_OK:
        msg = load().ptir_last_error(handle).decode(errors="replace") if handle else ""
        raise PtirError(rc, f"{what}: {msg}")
