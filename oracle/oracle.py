"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes front end of ``oracle/liboracle.so``, the CPU restatement of PTIR's Gaussian-field path
tracer (``oracle/oracle.cpp``). Only the tests, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` import this module; the shipped library never does.

All array arguments are numpy float32 (C-contiguous) in the layouts of the reference's
``OptixTracer.trace`` (threedgptir_tracer/src/optixTracer.cpp:909-1013).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class _Config(C.Structure):
    _fields_ = [
        ("kernel_degree", C.c_int),
        ("min_response", C.c_float),
        ("density_clamping", C.c_int),
        ("sph_max_coeffs", C.c_int),
        ("enable_normals", C.c_int),
        ("enable_hitcounts", C.c_int),
        ("enable_mis", C.c_int),
        ("enable_metallic", C.c_int),
        ("visualize_lights", C.c_int),
        ("draw_order", C.c_int),
    ]


_FP = C.POINTER(C.c_float)


class _Scene(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("bpos", _FP), ("brot", _FP), ("bscl", _FP), ("bdns", _FP),
        ("density", _FP), ("material", _FP), ("sph", _FP), ("snrm", _FP),
        ("env", _FP), ("eh", C.c_int), ("ew", C.c_int),
        ("alias", _FP), ("ah", C.c_int), ("aw", C.c_int),
        ("ray_to_world", _FP),
        ("ray_ori", _FP), ("ray_dir", _FP),
        ("nz", C.c_int), ("h", C.c_int), ("w", C.c_int),
        ("frame", C.c_uint),
        ("sph_degree", C.c_int),
        ("min_transmittance", C.c_float),
        ("max_bounces", C.c_uint),
        ("render_opts", C.c_uint),
        ("lights", _FP), ("light_table", _FP), ("mesh_vertices", _FP), ("mesh_triangles", C.POINTER(C.c_int)),
        ("mesh_lights", _FP), ("mesh_tri_table", _FP),
        ("num_lights", C.c_int), ("light_entries", C.c_int), ("num_mesh_vertices", C.c_int),
        ("num_mesh_triangles", C.c_int), ("num_mesh_lights", C.c_int), ("mesh_tri_cols", C.c_int),
    ]


class _FwdOut(C.Structure):
    _fields_ = [(k, _FP) for k in (
        "radiance", "density", "hit", "hit2", "distortion", "normal", "snormal", "material",
        "hits_count", "pbr", "light", "components", "visibility")] + [("path_sig", C.POINTER(C.c_uint32))]


class _BwdIn(C.Structure):
    _fields_ = [(k, _FP) for k in ("pbr", "light", "pbr_grad", "light_grad", "material_grad")]


class Stats(C.Structure):
    _fields_ = [(k, C.c_ulonglong) for k in (
        "segments", "trace_calls", "candidates", "accepted", "env_lookups", "replay_segments")]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


def build(reference_root: str | None = None) -> str:
    """Compile liboracle.so and libptir_kat.so, and with a reference checkout (the argument, else
    $PTIR_REFERENCE_ROOT) the binaries of oracle/_ref compiled from its sources."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    ref = reference_root or os.environ.get("PTIR_REFERENCE_ROOT")
    if ref and os.path.isdir(os.path.join(ref, "threedgptir_tracer")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={os.path.abspath(ref)}"], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.POINTER
        L.orc_trace_f64.argtypes = [P(_Config), P(_Scene), P(_FwdOut), C.c_int, C.c_longlong, P(Stats)]
        L.orc_trace_f32.argtypes = [P(_Config), P(_Scene), P(_FwdOut), C.c_int, C.c_longlong, P(Stats)]
        L.orc_trace_bwd_f64.argtypes = [P(_Config), P(_Scene), P(_BwdIn), P(C.c_double), P(C.c_double), C.c_int,
                                        C.c_longlong, P(Stats)]
        L.orc_trace_bwd_f32.argtypes = [P(_Config), P(_Scene), P(_BwdIn), P(C.c_double), P(C.c_double), C.c_int,
                                        C.c_longlong, P(Stats)]
        L.orc_trace_candidates.argtypes = [P(_Config), P(_Scene), C.c_int, _FP, _FP, _FP, P(C.c_uint), P(C.c_double)]
        L.orc_instances.argtypes = [P(_Config), P(_Scene), P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double)]
        L.orc_sampler_stream.argtypes = [C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, P(C.c_uint)]
        L.orc_launch_seed.argtypes = [C.c_uint, C.c_uint, C.c_uint, C.c_uint]
        L.orc_launch_seed.restype = C.c_ulonglong
        L.orc_num_threads.restype = C.c_int
        L.orc_light_samples.argtypes = [P(_Config), P(_Scene), C.c_int, _FP, P(C.c_double), P(C.c_double)]
        L.orc_kat.argtypes = [P(_Config), P(_Scene), C.c_char_p, C.c_int, _FP, P(C.c_double), P(C.c_double), C.c_int]
        _LIB = L
    return _LIB


@dataclass
class OracleConfig:
    """The tracer construction options the reference bakes in as JIT defines
    (optixTracer.cpp:240-272)."""

    kernel_degree: int = 4
    min_response: float = 0.0113
    density_clamping: bool = True
    sph_degree_max: int = 3
    enable_normals: bool = True
    enable_hitcounts: bool = True
    enable_mis: bool = True
    enable_metallic: bool = False
    visualize_lights: bool = False
    draw_order: int = 0

    def _c(self) -> _Config:
        return _Config(self.kernel_degree, self.min_response, int(self.density_clamping),
                       (self.sph_degree_max + 1) ** 2, int(self.enable_normals), int(self.enable_hitcounts),
                       int(self.enable_mis), int(self.enable_metallic), int(self.visualize_lights), self.draw_order)


def _f(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_FP)


class _Keep:
    """Holds converted arrays alive while a ctypes call runs."""

    def __init__(self):
        self.items = []

    def f32(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
        self.items.append(a)
        return a


def _scene(keep: _Keep, s: dict) -> _Scene:
    """Build the C scene from a dict of numpy arrays (see tests/scenes.py for the keys)."""
    g = lambda k: keep.f32(s.get(k))  # noqa: E731
    dens = g("density")
    n = 0 if dens is None else dens.shape[0]
    env = g("environment")
    eh = ew = 0
    if env is not None and env.ndim == 3 and env.shape[0] > 0 and env.shape[1] > 0 and env.shape[2] == 4:
        eh, ew = env.shape[0], env.shape[1]
    else:
        env = None
    alias = g("alias_table")
    ah = aw = 0
    if alias is not None and alias.ndim == 3 and alias.shape[0] == 3 and alias.size > 0:
        ah, aw = alias.shape[1], alias.shape[2]
    else:
        alias = None
    ori, dirs = g("ray_ori"), g("ray_dir")
    nz, h, w = ori.shape[0], ori.shape[1], ori.shape[2]
    t = keep.f32(np.asarray(s.get("ray_to_world", np.eye(4, dtype=np.float32))).reshape(-1, 4, 4)[0][:3].reshape(12))
    sc = _Scene()
    sc.n = n
    for k, key in (("bpos", "build_pos"), ("brot", "build_rot"), ("bscl", "build_scl"), ("bdns", "build_dns")):
        setattr(sc, k, _f(g(key)))
    sc.density = _f(dens)
    sc.material = _f(g("material"))
    sc.sph = _f(g("sph"))
    sc.snrm = _f(g("shading_normal"))
    sc.env, sc.eh, sc.ew = _f(env), eh, ew
    sc.alias, sc.ah, sc.aw = _f(alias), ah, aw
    sc.ray_to_world = _f(t)
    sc.ray_ori, sc.ray_dir = _f(ori), _f(dirs)
    sc.nz, sc.h, sc.w = nz, h, w
    sc.frame = int(s.get("frame", 0))
    sc.sph_degree = int(s.get("sph_degree", 3))
    sc.min_transmittance = float(s.get("min_transmittance", 0.001))
    sc.max_bounces = int(s.get("max_bounces", 3))
    sc.render_opts = int(s.get("render_opts", 0))
    # punctual and area lights (LightBuffers): 2-D row-major tables, absent or empty = none
    tables = (("lights", "lights", "num_lights", 0), ("light_alias_table", "light_table", "light_entries", 1),
              ("mesh_light_vertices", "mesh_vertices", "num_mesh_vertices", 0),
              ("mesh_lights", "mesh_lights", "num_mesh_lights", 0),
              ("mesh_light_triangle_alias_table", "mesh_tri_table", "mesh_tri_cols", 1))
    for key, field, count, axis in tables:
        a = g(key)
        if a is not None and a.ndim == 2 and a.size > 0:
            setattr(sc, field, _f(a))
            setattr(sc, count, int(a.shape[axis]))
    tris = s.get("mesh_light_triangles")
    if tris is not None and np.asarray(tris).size > 0:
        tris = np.ascontiguousarray(np.asarray(tris, dtype=np.int32))
        keep.items.append(tris)
        sc.mesh_triangles = tris.ctypes.data_as(C.POINTER(C.c_int))
        sc.num_mesh_triangles = int(tris.shape[0])
    return sc


FWD_KEYS = ("radiance", "density", "hit", "hit2", "distortion", "normal", "snormal", "material", "hits_count",
            "pbr", "light", "components")
_FWD_CH = {"radiance": 3, "density": 1, "hit": 2, "hit2": 1, "distortion": 1, "normal": 3, "snormal": 3,
           "material": 5, "hits_count": 1, "pbr": 3, "light": 3, "components": 6}


def trace(cfg: OracleConfig, scene: dict, precision: str = "f64", threads: int = 0, stride: int = 1):
    """Forward trace of every `stride`-th path (flat launch index li % stride == 0; the others'
    outputs stay zero). Returns (dict of outputs [nz,h,w,C] float32, visibility [n], Stats); the
    dict also holds 'path_sig' [nz,h,w] uint32, each path's decision signature (the hash the GPU
    tracer writes to its path_signature output)."""
    keep = _Keep()
    sc = _scene(keep, scene)
    shape = (sc.nz, sc.h, sc.w)
    outs = {k: np.zeros(shape + (_FWD_CH[k],), np.float32) for k in FWD_KEYS}
    outs["components"] = outs["components"].reshape(shape + (2, 3))
    vis = np.zeros((max(sc.n, 1),), np.float32)
    sig = np.zeros(shape, np.uint32)
    fo = _FwdOut(*[_f(outs[k]) for k in FWD_KEYS], _f(vis), sig.ctypes.data_as(C.POINTER(C.c_uint32)))
    st = Stats()
    c = cfg._c()
    if precision == "f64":
        rc = lib().orc_trace_f64(C.byref(c), C.byref(sc), C.byref(fo), threads, stride, C.byref(st))
    else:
        rc = lib().orc_trace_f32(C.byref(c), C.byref(sc), C.byref(fo), threads, stride, C.byref(st))
    assert rc == 0
    outs["path_sig"] = sig
    return outs, vis[: sc.n], st


def trace_bwd(cfg: OracleConfig, scene: dict, fwd: dict, grads: dict, precision: str = "f64", threads: int = 0,
              stride: int = 1):
    """Backward (path replay) of every `stride`-th path. ``fwd`` holds 'pbr' and 'light'; ``grads``
    holds 'pbr', 'light', 'material' output gradients. Returns (material_grad [n,5] f64, env_grad
    [eh,ew,4] f64, Stats)."""
    keep = _Keep()
    sc = _scene(keep, scene)
    bi = _BwdIn(_f(keep.f32(fwd["pbr"])), _f(keep.f32(fwd["light"])), _f(keep.f32(grads.get("pbr"))),
                _f(keep.f32(grads.get("light"))), _f(keep.f32(grads.get("material"))))
    mg = np.zeros((max(sc.n, 1), 5), np.float64)
    eg = np.zeros((max(sc.eh, 1), max(sc.ew, 1), 4), np.float64)
    st = Stats()
    c = cfg._c()
    P = C.POINTER(C.c_double)
    if precision == "f64":
        rc = lib().orc_trace_bwd_f64(C.byref(c), C.byref(sc), C.byref(bi), mg.ctypes.data_as(P), eg.ctypes.data_as(P),
                                     threads, stride, C.byref(st))
    else:
        rc = lib().orc_trace_bwd_f32(C.byref(c), C.byref(sc), C.byref(bi), mg.ctypes.data_as(P), eg.ctypes.data_as(P),
                                     threads, stride, C.byref(st))
    assert rc == 0
    return mg[: sc.n], eg[: sc.eh, : sc.ew], st


def candidates(cfg: OracleConfig, scene: dict, rays: np.ndarray, tmin: np.ndarray, tend: np.ndarray):
    """The 16 nearest candidates of single trace() calls. Returns (ids [m,16] uint32, t [m,16] f64)."""
    keep = _Keep()
    sc = _scene(keep, scene)
    rays = keep.f32(rays)
    tmin, tend = keep.f32(tmin), keep.f32(tend)
    m = rays.shape[0]
    ids = np.zeros((m, 16), np.uint32)
    ts = np.zeros((m, 16), np.float64)
    c = cfg._c()
    rc = lib().orc_trace_candidates(C.byref(c), C.byref(sc), m, _f(rays), _f(tmin), _f(tend),
                                    ids.ctypes.data_as(C.POINTER(C.c_uint)), ts.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    return ids, ts


def instances(cfg: OracleConfig, scene: dict):
    """Scene AABB [6], kernel scale [n], per-Gaussian world AABB lo/hi [n,3] (all f64)."""
    keep = _Keep()
    sc = _scene(keep, scene)
    n = sc.n
    aabb = np.zeros(6, np.float64)
    ks = np.zeros(max(n, 1), np.float64)
    lo = np.zeros((max(n, 1), 3), np.float64)
    hi = np.zeros((max(n, 1), 3), np.float64)
    P = C.POINTER(C.c_double)
    c = cfg._c()
    lib().orc_instances(C.byref(c), C.byref(sc), aabb.ctypes.data_as(P), ks.ctypes.data_as(P), lo.ctypes.data_as(P),
                        hi.ctypes.data_as(P))
    return aabb, ks[:n], lo[:n], hi[:n]


def sampler_stream(x: int, y: int, z: int, frame: int, count: int) -> np.ndarray:
    out = np.zeros(count, np.uint32)
    lib().orc_sampler_stream(x, y, z, frame, count, out.ctypes.data_as(C.POINTER(C.c_uint)))
    return out


def launch_seed(x: int, y: int, z: int, frame: int) -> int:
    return int(lib().orc_launch_seed(x, y, z, frame))


def light_samples(cfg: OracleConfig, scene: dict, positions: np.ndarray, frame: int = 0):
    """One light sample per position (sample i from launch stream (i, 0, 0, frame)). Returns
    (wi [m,3], Li [m,3], pdf [m], dist [m], type [m] int, pdf of wi under the light sampler [m]), FP64."""
    keep = _Keep()
    sc = _scene(keep, scene)
    sc.frame = int(frame)
    pos = keep.f32(positions).reshape(-1, 3)
    m = pos.shape[0]
    out = np.zeros((m, 9), np.float64)
    ev = np.zeros(m, np.float64)
    P = C.POINTER(C.c_double)
    c = cfg._c()
    rc = lib().orc_light_samples(C.byref(c), C.byref(sc), m, _f(pos), out.ctypes.data_as(P), ev.ctypes.data_as(P))
    assert rc == 0
    return out[:, :3], out[:, 3:6], out[:, 6], out[:, 7], out[:, 8].astype(np.int64), ev


KAT_COLUMNS = {"process_hit": 18, "intersect": 2, "brdf_sample": 7, "brdf_eval": 4, "brdf_grads": 19,
               "env_lookup": 4, "env_bwd": 6, "env_sample": 4, "light_sample": 9, "light_pdf": 1}


def kat(cfg: OracleConfig, scene: dict, name: str, inputs: np.ndarray, precision: str = "f64"):
    """The oracle's evaluation of one reference function on known-answer inputs laid out as
    oracle/ref_device_kat.cu lays them out, in FP64 or ("f32") its FP32 instantiation. Returns
    (outputs [n, KAT_COLUMNS[name]] f64, environment gradient [eh, ew, 4] f64 of "env_bwd")."""
    keep = _Keep()
    s = dict(scene)
    s.setdefault("ray_ori", np.zeros((1, 1, 1, 3), np.float32))
    s.setdefault("ray_dir", np.zeros((1, 1, 1, 3), np.float32))
    sc = _scene(keep, s)
    x = keep.f32(inputs)
    n = x.shape[0]
    out = np.zeros((n, KAT_COLUMNS[name]), np.float64)
    eg = np.zeros((max(sc.eh, 1), max(sc.ew, 1), 4), np.float64)
    P = C.POINTER(C.c_double)
    rc = lib().orc_kat(C.byref(cfg._c()), C.byref(sc), name.encode(), n, _f(x), out.ctypes.data_as(P),
                       eg.ctypes.data_as(P), 1 if precision == "f32" else 0)
    assert rc == 0, name
    return out, eg[: sc.eh, : sc.ew]


def num_threads() -> int:
    return int(lib().orc_num_threads())
