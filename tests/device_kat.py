"""Shared helpers of the known-answer tests on tests/golden/device_kat.npz (vectors of the
reference's own device functions, compiled from its headers with its NVRTC options and run on a
GPU by tests/golden/make_device_golden.py)."""
from __future__ import annotations

import os

import numpy as np

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "device_kat.npz")
LIGHT_KEYS = ("lights", "light_alias_table", "mesh_light_vertices", "mesh_light_triangles", "mesh_lights",
              "mesh_light_triangle_alias_table")

# (entry, fixture key, output columns compared, scene)
CASES = (
    ("process_hit", "process_hit", 18, "particles"),
    ("intersect", "intersect", 2, None),
    ("brdf_sample", "brdf_sample", 7, None),
    ("brdf_eval", "brdf_eval", 4, None),
    ("brdf_grads", "brdf_grads", 19, None),
    ("env_lookup", "env_lookup_equirect", 4, "equirect"),
    ("env_lookup", "env_lookup_cube", 4, "cube"),
    ("env_bwd", "env_bwd_equirect", 6, "equirect"),
    ("env_bwd", "env_bwd_cube", 6, "cube"),
    ("env_sample", "env_sample_equirect", 4, "equirect"),
    ("env_sample", "env_sample_cube", 4, "cube"),
    ("light_sample", "light_sample", 9, "lights"),
    ("light_pdf", "light_pdf", 1, "lights"),
)


def load():
    return dict(np.load(FIXTURE))


def oracle_scene(g: dict, scene: str | None) -> dict:
    """The oracle scene dict of a fixture scene."""
    if scene == "particles":
        d = g["particles_density"]
        return dict(density=d, material=g["particles_material"], sph=g["particles_sph"],
                    shading_normal=g["particles_shading_normal"], build_pos=np.ascontiguousarray(d[:, 0:3]),
                    build_rot=np.ascontiguousarray(d[:, 4:8]), build_scl=np.ascontiguousarray(d[:, 8:11]),
                    build_dns=np.ascontiguousarray(d[:, 3:4]))
    if scene in ("equirect", "cube"):
        return dict(environment=g[f"env_{scene}"], alias_table=g[f"alias_{scene}"])
    if scene == "lights":
        s = dict(environment=g["lightscene_env"], alias_table=g["lightscene_alias"])
        s.update({k: g[f"lightscene_{k}"] for k in LIGHT_KEYS})
        return s
    return {}


EPS32 = 2.0 ** -24

# Outputs that are forward differences of float evaluations over eps = 1e-3: the roughness
# derivative of the sampled direction (material.cuh:30,362-375) and the direction gradient of an
# environment lookup (environment.cuh:16,421-445). Their rounding error is that of the two
# evaluations times 1 / eps, so they are compared as vectors (fd_report).
FD_COLUMNS = {"brdf_grads": slice(12, 15), "env_bwd": slice(3, 6)}


def value_columns(entry: str, cols: int) -> list:
    fd = FD_COLUMNS.get(entry)
    return [c for c in range(cols) if fd is None or not fd.start <= c < fd.stop]


def case_rtol(entry: str, x: np.ndarray, rtol: float) -> np.ndarray:
    """Per-case relative tolerance: `rtol`, widened for the BRDF functions by the float
    conditioning of the GGX sampling and distribution at roughness r: 1 + (alpha^2 - 1) u with
    alpha = max(r, 0.05)^2 keeps only log2(1 / alpha^2) fewer bits (material.cuh:26-27,230-286), so
    the float result carries about eps32 / alpha^2 of relative error."""
    if entry.startswith("brdf"):
        a2 = np.maximum(x[:, 10].astype(np.float64), 0.05) ** 4
        return rtol + 4.0 * EPS32 / a2
    return np.full(x.shape[0], rtol)


def close(x, ref, atol, rtol):
    """Per case: every column within atol + rtol * |ref| (rtol a scalar or one per case)."""
    x, ref = np.asarray(x, np.float64), np.asarray(ref, np.float64)
    rtol = np.asarray(rtol, np.float64)
    if rtol.ndim == 1:
        rtol = rtol[:, None]
    return np.all(np.abs(x - ref) <= atol + rtol * np.abs(ref), axis=-1)


def fd_report(out, ref) -> dict:
    """Finite-difference outputs as vectors: relative L2 and cosine over all cases, and the share of
    cases within 1e-4 + 1e-2 |ref| (vector norms)."""
    a, b = np.asarray(out, np.float64), np.asarray(ref, np.float64)
    nb = np.linalg.norm(b)
    rel = float(np.linalg.norm(a - b) / max(nb, 1e-30))
    cos = float((a * b).sum() / max(np.linalg.norm(a) * nb, 1e-30))
    share = float(np.mean(np.linalg.norm(a - b, axis=1) <= 1e-4 + 1e-2 * np.linalg.norm(b, axis=1)))
    return dict(rel_l2=rel, cos=cos, share=share)


class PtirKat:
    """The tracer's device functions behind the same entries (oracle/libptir_kat.so), on torch CUDA
    tensors."""

    def __init__(self):
        import ctypes as C

        path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "libptir_kat.so")
        self.lib = C.CDLL(path)
        self.C = C

    def set_scene(self, g: dict, scene: str | None):
        import torch

        C = self.C
        s = oracle_scene(g, scene)
        t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in s.items() if isinstance(v, np.ndarray)}
        self._keep = t
        p = lambda k: C.c_void_p(t[k].data_ptr() if k in t and t[k].numel() else 0)  # noqa: E731
        dim = lambda k, ax: C.c_int(int(t[k].shape[ax]) if k in t else 0)  # noqa: E731
        env = "environment"
        self.lib.ptirkat_set_scene(p(env), dim(env, 0), dim(env, 1), p("alias_table"), dim("alias_table", 1),
                                   dim("alias_table", 2), p("lights"), dim("lights", 0), p("light_alias_table"),
                                   dim("light_alias_table", 1), p("mesh_light_vertices"), dim("mesh_light_vertices", 0),
                                   p("mesh_light_triangles"), dim("mesh_light_triangles", 0), p("mesh_lights"),
                                   dim("mesh_lights", 0), p("mesh_light_triangle_alias_table"),
                                   dim("mesh_light_triangle_alias_table", 1))
        return t

    def run(self, entry: str, g: dict, scene: str | None, x: np.ndarray, cols: int):
        """(outputs [n, cols] numpy, environment gradient or None)."""
        import torch

        C = self.C
        t = self.set_scene(g, scene)
        xi = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
        n = xi.shape[0]
        width = {"process_hit": 18, "light_sample": 9}.get(entry, cols)
        y = torch.zeros((n, width), dtype=torch.float32, device="cuda")
        args = [C.c_int(n), C.c_void_p(xi.data_ptr()), C.c_void_p(y.data_ptr())]
        eg = None
        if entry == "process_hit":
            args += [C.c_void_p(t[k].data_ptr()) for k in ("density", "material", "sph", "shading_normal")]
            args += [C.c_float(0.0113), C.c_float(1.0 / 255.0), C.c_int(3)]
        elif entry == "env_bwd":
            env = t["environment"]
            eg = torch.zeros_like(env)
            args += [C.c_void_p(eg.data_ptr()), C.c_int(env.shape[0]), C.c_int(env.shape[1])]
        rc = getattr(self.lib, f"ptirkat_{entry}")(*args)
        assert rc == 0, entry
        return y.cpu().numpy(), (eg.cpu().numpy() if eg is not None else None)
