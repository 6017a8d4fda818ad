"""Small seeded scenes shared by the oracle and GPU tests."""
from __future__ import annotations

import numpy as np
import torch

from ptir_b200 import envmap, synthetic


def small_scene(n=2000, w=48, h=40, spp=1, views=1, max_bounces=3, env_hw=(32, 64), seed=0, sh_full=False,
                scale_range=(0.01, 0.08), frame=3, sh_degree=3, env=True, alias=True, cube=False, layout="uniform"):
    """Returns a dict of numpy float32 arrays in the tracer's layouts plus the scalars, ready for
    oracle.trace() and for to_torch()."""
    f = synthetic.make_field(n, seed=seed, layout=layout, scale_range=scale_range, sh_degree=sh_degree, sh_full=sh_full)
    eyes = synthetic.camera_positions(views, seed=seed)
    oris, dirs = [], []
    for v in range(views):
        o, d = synthetic.view_rays(w, h, spp, eyes[v])
        oris.append(o)
        dirs.append(d)
    # launch z = sample * views + view (the reference's spp expansion order)
    ori = torch.stack(oris, 1).reshape(spp * views, h, w, 3)
    dr = torch.stack(dirs, 1).reshape(spp * views, h, w, 3)
    s = dict(
        build_pos=f["pos"].numpy(), build_rot=f["rot"].numpy(), build_scl=f["scl"].numpy(), build_dns=f["dns"].numpy(),
        density=synthetic.density_tensor(f).numpy(), material=synthetic.material_tensor(f).numpy(),
        sph=f["sph"].numpy(), shading_normal=f["snrm"].numpy(),
        ray_ori=ori.numpy(), ray_dir=dr.numpy(), ray_to_world=np.eye(4, dtype=np.float32)[None],
        frame=frame, sph_degree=sh_degree, min_transmittance=0.001, max_bounces=max_bounces, render_opts=0,
    )
    if env:
        eh, ew = env_hw
        e = synthetic.make_environment(6 * ew if cube else eh, ew, seed=seed)
        s["environment"] = e.numpy()
        if alias:
            s["alias_table"] = envmap.pack(envmap.build(e, cube=cube)).numpy()
        else:
            s["alias_table"] = np.zeros((0,), np.float32)
    else:
        s["environment"] = np.zeros((0, 0, 4), np.float32)
        s["alias_table"] = np.zeros((0,), np.float32)
    return s


LIGHT_KEYS = ("lights", "light_alias_table", "mesh_light_vertices", "mesh_light_triangles", "mesh_lights",
              "mesh_light_triangle_alias_table")


def with_lights(s: dict, lights, environment=True) -> dict:
    """The scene with the packed tables of `lights` (point / sphere / mesh dicts) and a top-level
    light table that includes the scene's environment when `environment` is set and it has one."""
    from ptir_b200.lights import light_buffers

    env = s.get("environment")
    env_t = torch.from_numpy(env) if environment and env is not None and env.size > 0 else None
    lb = light_buffers(lights, environment=env_t)
    tables = dict(zip(LIGHT_KEYS, (t.numpy() for t in lb.tensors())))
    return dict(s, **tables)


def _light_tensors(S: dict) -> tuple:
    dev = S["density"].device
    empty = {"lights": (0, 9), "light_alias_table": (5, 0), "mesh_light_vertices": (0, 3),
             "mesh_light_triangles": (0, 3), "mesh_lights": (0, 8), "mesh_light_triangle_alias_table": (3, 0)}
    out = []
    for k in LIGHT_KEYS:
        if k in S:
            out.append(S[k])
        else:
            dt = torch.int32 if k == "mesh_light_triangles" else torch.float32
            out.append(torch.empty(empty[k], dtype=dt, device=dev))
    return tuple(out)


def to_torch(s: dict, device="cuda") -> dict:
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    return {k: (t(v) if isinstance(v, np.ndarray) else v) for k, v in s.items()}


def make_tracer(sph_degree=3, normals=True, hitcounts=True, mis=True, metallic=False, visualize=False,
                kernel_degree=4, min_response=0.0113, clamping=True, schedule="wavefront", chunk_tiles=0, kbuffer=16,
                **launch):
    from ptir_b200 import OptixTracer

    return OptixTracer("", "", "reference", "referenceBwd", "instances", kernel_degree, min_response, clamping,
                       sph_degree, normals, hitcounts, mis, metallic, visualize, schedule=schedule,
                       chunk_tiles=chunk_tiles, kbuffer=kbuffer, **launch)


def round_to(a: np.ndarray, storage: str) -> np.ndarray:
    """float32 values rounded to bf16 / fp16 (nearest even) and widened back, as the tracer's
    16-bit storage holds them."""
    a = np.ascontiguousarray(a, np.float32)
    if storage == "fp16":
        return a.astype(np.float16).astype(np.float32)
    if storage == "bf16":
        u = a.view(np.uint32).astype(np.uint64)
        u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
        return u.astype(np.uint32).view(np.float32)
    return a


ATTRIBUTES = ("build_pos", "build_rot", "build_scl", "build_dns", "density", "material", "sph", "shading_normal")


def round_scene(s: dict, storage: str) -> dict:
    """The scene as a tracer with 16-bit attribute storage sees it."""
    return dict(s, **{k: round_to(s[k], storage) for k in ATTRIBUTES})


def gpu_trace(tr, S: dict, build=True, rebuild=True):
    """Run build_bvh + trace on torch CUDA scene S (from to_torch). Returns the 13-tuple."""
    if build:
        tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], rebuild, True)
    return tr.trace(S["frame"], S["ray_to_world"], S["ray_ori"], S["ray_dir"], S["density"], S["material"], S["sph"],
                    S["shading_normal"], S["environment"], S["alias_table"], *_light_tensors(S), S["render_opts"],
                    S["sph_degree"], S["min_transmittance"], S["max_bounces"])


def gpu_trace_bwd(tr, S: dict, fwd, pbr_grad, light_grad=None, material_grad=None):
    (rad, dns, hit, hit2, dist, nrm, snrm, mat, hits, vis, pbr, light, comps) = fwd
    z = lambda t: torch.zeros_like(t)  # noqa: E731
    if light_grad is None:
        light_grad = z(light)
    if material_grad is None:
        material_grad = z(mat)
    return tr.trace_bwd(S["frame"], S["ray_to_world"], S["ray_ori"], S["ray_dir"], rad, dns, hit, hit2, dist, nrm, snrm,
                        mat, pbr, light, S["density"], S["material"], S["sph"], S["shading_normal"], S["environment"],
                        S["alias_table"], *_light_tensors(S), z(rad), z(dns), z(hit), z(hit2), z(dist), z(nrm), z(snrm),
                        material_grad, pbr_grad, light_grad, S["render_opts"], S["sph_degree"], S["min_transmittance"],
                        S["max_bounces"])


def workload_scene(name: str, view: int = 0, frame: int = 0) -> dict:
    """The scene dict (as small_scene returns) of one view of a named benchmark workload
    (ptir_b200/synthetic.py), with the benchmark's generator, camera, environment and alias table."""
    wl = synthetic.workload(name)
    f = synthetic.make_field(wl.n, seed=wl.seed, layout=wl.layout, scale_range=wl.scale_range, sh_full=wl.sh_full)
    w, h, spp = wl.views[view]
    eye = synthetic.camera_positions(len(wl.views), seed=wl.seed)[view]
    o, d = synthetic.view_rays(w, h, spp, eye)
    env = synthetic.make_environment(*wl.env_hw, seed=wl.seed)
    return dict(
        build_pos=f["pos"].numpy(), build_rot=f["rot"].numpy(), build_scl=f["scl"].numpy(), build_dns=f["dns"].numpy(),
        density=synthetic.density_tensor(f).numpy(), material=synthetic.material_tensor(f).numpy(),
        sph=f["sph"].numpy(), shading_normal=f["snrm"].numpy(), ray_ori=o.numpy(), ray_dir=d.numpy(),
        ray_to_world=np.eye(4, dtype=np.float32)[None], frame=frame, sph_degree=3, min_transmittance=0.001,
        max_bounces=wl.max_bounces, render_opts=0, environment=env.numpy(),
        alias_table=envmap.pack(envmap.build(env)).numpy())
