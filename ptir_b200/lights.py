"""Light tables for next-event estimation (the input producer of the tracer's light sampler).

Builds the packed tensors the tracer reads (the reference's LightBuffers,
threedgptir_tracer/tracer.py:40-119) from light descriptions, following the reference's
threedgrut/model/light.py:

    pack_lights                 [L, 9]  type, position / center xyz, radius, radiance rgb, two_sided
                                        (Light.pack_lights, light.py:225-266)
    pack_mesh_lights            vertices [V, 3], triangles [T, 3] (global vertex indices), params
                                [M, 8], triangle alias table [3, T], powers [M] (light.py:1769-1859)
    build_light_alias_table     [5, E]  Vose table over the environment, point, sphere and mesh
                                lights weighted by estimated power (light.py:1480-1584)

Light descriptions are dicts: {"type": "point", "position", "intensity"},
{"type": "sphere", "center", "radius", "radiance", "two_sided"} and
{"type": "mesh", "vertices", "triangles", "radiance", "two_sided"}. Powers are Rec.709 luminance
times emitting area (4 pi r^2 for spheres, twice the area for two-sided meshes); the environment's
is its luminance integrated over solid angle. The alias construction is the float64 Vose of the
environment table (envmap.vose).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .envmap import LUMINANCE, _solid_angles_cube, _solid_angles_equirect, vose

LIGHT_TYPE_ENV, LIGHT_TYPE_POINT, LIGHT_TYPE_SPHERE, LIGHT_TYPE_MESH = 0, 1, 2, 3
PACKED_LIGHT_SIZE = 9
PACKED_MESH_LIGHT_SIZE = 8


def _luminance(rgb: torch.Tensor) -> torch.Tensor:
    return torch.sum(rgb[..., :3] * rgb.new_tensor(LUMINANCE), dim=-1)


def _vec3(v, name: str) -> torch.Tensor:
    t = torch.as_tensor(v, dtype=torch.float32).reshape(-1)
    if t.numel() != 3:
        raise ValueError(f"{name} must have 3 components")
    return t


def _pack_one(light: dict) -> torch.Tensor:
    kind = str(light.get("type", "")).lower()
    if kind == "point":
        pos = _vec3(light.get("position", (0.0, 0.0, 0.0)), "position")
        inten = _vec3(light.get("intensity", light.get("radiance", (1.0, 1.0, 1.0))), "intensity")
        if bool((inten < 0).any()):
            raise ValueError("intensity must be non-negative")
        z = torch.zeros(1)
        return torch.cat([torch.tensor([float(LIGHT_TYPE_POINT)]), pos, z, inten, z])
    if kind == "sphere":
        center = _vec3(light.get("center", (0.0, 0.0, 0.0)), "center")
        radius = float(light.get("radius", 1.0))
        rad = _vec3(light.get("radiance", (1.0, 1.0, 1.0)), "radiance")
        if radius <= 0.0:
            raise ValueError("radius must be positive")
        if bool((rad < 0).any()):
            raise ValueError("radiance must be non-negative")
        two = 1.0 if light.get("two_sided", False) else 0.0
        return torch.cat([torch.tensor([float(LIGHT_TYPE_SPHERE)]), center, torch.tensor([radius]), rad,
                          torch.tensor([two])])
    raise NotImplementedError(f"packed lights hold point and sphere lights, got '{kind}'")


def pack_lights(lights, device=None) -> torch.Tensor:
    """[L, 9] float32 table of point and sphere lights (a ready [L, 9] tensor passes through)."""
    if lights is None:
        return torch.empty((0, PACKED_LIGHT_SIZE), dtype=torch.float32, device=device)
    if isinstance(lights, torch.Tensor):
        t = lights.to(device=device, dtype=torch.float32)
        if t.numel() == 0:
            return torch.empty((0, PACKED_LIGHT_SIZE), dtype=torch.float32, device=device)
        if t.dim() != 2 or t.shape[1] != PACKED_LIGHT_SIZE:
            raise ValueError(f"packed lights must be [N, {PACKED_LIGHT_SIZE}], got {tuple(t.shape)}")
        return t.contiguous()
    rows = [_pack_one(light) for light in lights]
    if not rows:
        return torch.empty((0, PACKED_LIGHT_SIZE), dtype=torch.float32, device=device)
    return torch.stack(rows).to(device=device).contiguous()


def estimate_light_power(packed: torch.Tensor) -> torch.Tensor:
    """Power of each packed light: luminance of the intensity (point) or of the radiance times
    4 pi r^2 (sphere); 0 for other types."""
    packed = torch.as_tensor(packed, dtype=torch.float32)
    if packed.numel() == 0:
        return packed.new_empty((0,))
    powers = packed.new_zeros((packed.shape[0],))
    kinds = packed[:, 0].round().to(torch.int64)
    point = kinds == LIGHT_TYPE_POINT
    if bool(point.any()):
        powers[point] = _luminance(torch.clamp(packed[point, 5:8], min=0.0))
    sphere = kinds == LIGHT_TYPE_SPHERE
    if bool(sphere.any()):
        r = torch.clamp(packed[sphere, 4], min=0.0)
        powers[sphere] = _luminance(torch.clamp(packed[sphere, 5:8], min=0.0)) * (4.0 * torch.pi * r * r)
    return powers.contiguous()


def _triangle_areas(vertices: torch.Tensor, triangles: torch.Tensor) -> torch.Tensor:
    tv = vertices[triangles.to(torch.long)]
    areas = 0.5 * torch.linalg.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0], dim=-1).norm(dim=-1)
    return torch.where(torch.isfinite(areas) & (areas > 0.0), areas, torch.zeros_like(areas))


def _alias(weights: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    prob, alias = vose(weights.detach().cpu().numpy())
    return torch.from_numpy(prob), torch.from_numpy(alias.astype(np.int32))


@dataclass(frozen=True)
class MeshLightPack:
    vertices: torch.Tensor              # [V, 3]
    triangles: torch.Tensor             # [T, 3] int32, global vertex indices
    params: torch.Tensor                # [M, 8]
    triangle_alias_table: torch.Tensor  # [3, T]: prob, alias (local to its mesh), area pdf
    powers: torch.Tensor                # [M]


def pack_mesh_lights(meshes, device=None) -> MeshLightPack:
    """Concatenate triangle-mesh lights; meshes without area are left out."""
    f32 = dict(dtype=torch.float32, device=device)
    verts, tris, params, prob, alias, pdf, powers = [], [], [], [], [], [], []
    v_off = t_off = 0
    for m in meshes or ():
        v = torch.as_tensor(m["vertices"], dtype=torch.float32).reshape(-1, 3)
        t = torch.as_tensor(m["triangles"]).reshape(-1, 3).to(torch.int64)
        if t.numel() == 0 or v.shape[0] == 0:
            raise ValueError("a mesh light needs vertices and triangles")
        if bool((t < 0).any()) or bool((t >= v.shape[0]).any()):
            raise ValueError("triangle index outside the vertex range")
        t = t.to(torch.int32)
        rad = _vec3(m.get("radiance", (1.0, 1.0, 1.0)), "radiance")
        if bool((rad < 0).any()):
            raise ValueError("radiance must be non-negative")
        two = bool(m.get("two_sided", False))
        areas = _triangle_areas(v, t)
        total = areas.sum()
        if not bool(torch.isfinite(total)) or float(total) <= 0.0:
            continue
        p, a = _alias(areas)
        area_pdf = torch.where(areas > 0.0, (areas / total) / torch.clamp(areas, min=torch.finfo(areas.dtype).tiny),
                               torch.zeros_like(areas))
        verts.append(v)
        tris.append(t + v_off)
        params.append(torch.tensor([float(t_off), float(t.shape[0]), float(v_off), float(v.shape[0]),
                                    float(rad[0]), float(rad[1]), float(rad[2]), 1.0 if two else 0.0]))
        prob.append(p)
        alias.append(a.to(torch.float32))
        pdf.append(area_pdf.to(torch.float32))
        powers.append(_luminance(torch.clamp(rad, min=0.0)) * total.reshape(1)[0] * (2.0 if two else 1.0))
        v_off += v.shape[0]
        t_off += t.shape[0]
    if not params:
        return MeshLightPack(torch.empty((0, 3), **f32), torch.empty((0, 3), dtype=torch.int32, device=device),
                             torch.empty((0, PACKED_MESH_LIGHT_SIZE), **f32), torch.empty((3, 0), **f32),
                             torch.empty((0,), **f32))
    return MeshLightPack(torch.cat(verts).to(device).contiguous(), torch.cat(tris).to(device).contiguous(),
                         torch.stack(params).to(device).contiguous(),
                         torch.stack([torch.cat(prob), torch.cat(alias), torch.cat(pdf)]).to(device).contiguous(),
                         torch.stack(powers).reshape(-1).to(device).contiguous())


def environment_power(environment: torch.Tensor | None, environment_type: str = "2d") -> torch.Tensor | None:
    """Luminance of an [H, W, C>=3] environment integrated over solid angle (full resolution);
    None when absent or dark."""
    if environment is None or environment.numel() == 0:
        return None
    env = environment.detach().to("cpu", torch.float32)
    rgb = env[..., :3]
    rgb = torch.where(torch.isfinite(rgb) & (rgb > 0.0), rgb, torch.zeros_like(rgb))
    lum = torch.sum(rgb * rgb.new_tensor(LUMINANCE), dim=-1)
    h, w = lum.shape
    if str(environment_type).lower() == "cube":
        if h != 6 * w:
            raise ValueError(f"cube map environment must be [6N, N, C], got H={h}, W={w}")
        sa = _solid_angles_cube(w)
    else:
        sa = _solid_angles_equirect(h, w)
    power = (lum * sa).sum()
    if not bool(torch.isfinite(power)) or float(power) <= 0.0:
        return None
    return power


def build_light_alias_table(environment=None, environment_type: str = "2d", lights=None, mesh_powers=None,
                            environment_index: int = 0, device=None) -> torch.Tensor:
    """[5, E] float32 top-level table (prob, alias, type, index, selection pdf) over the lights
    with finite positive power; [5, 0] when there is none (the tracer then samples the environment
    alone)."""
    types, index, weights = [], [], []
    env_power = environment_power(environment, environment_type)
    if env_power is not None:
        types.append(LIGHT_TYPE_ENV)
        index.append(int(environment_index))
        weights.append(env_power)
    packed = pack_lights(lights)
    for i, pw in enumerate(estimate_light_power(packed.cpu())):
        if bool(torch.isfinite(pw)) and float(pw) > 0.0:
            types.append(int(float(packed[i, 0]) + 0.5))
            index.append(i)
            weights.append(pw)
    if mesh_powers is not None:
        for i, pw in enumerate(torch.as_tensor(mesh_powers, dtype=torch.float32).reshape(-1).cpu()):
            if bool(torch.isfinite(pw)) and float(pw) > 0.0:
                types.append(LIGHT_TYPE_MESH)
                index.append(i)
                weights.append(pw)
    empty = torch.empty((5, 0), dtype=torch.float32, device=device)
    if not weights:
        return empty
    w = torch.stack([torch.as_tensor(x, dtype=torch.float32).cpu() for x in weights])
    total = w.sum()
    if not bool(torch.isfinite(total)) or float(total) <= 0.0:
        return empty
    prob, alias = _alias(w)
    select = (w / total).to(torch.float32)
    table = torch.stack([prob, alias.to(torch.float32), torch.tensor(types, dtype=torch.float32),
                         torch.tensor(index, dtype=torch.float32), select])
    return table.to(device).contiguous()


def light_buffers(lights=None, environment=None, environment_type: str = "2d", device=None):
    """The six tracer tables for a list of light descriptions (point, sphere and mesh dicts) and an
    optional environment, assembled as the reference's renderer does (threedgrut/render.py:195-240).
    Returns ptir_b200.tracer.LightBuffers."""
    from .tracer import LightBuffers

    lights = list(lights or ())
    meshes = [m for m in lights if str(m.get("type", "")).lower() == "mesh"]
    analytic = [m for m in lights if str(m.get("type", "")).lower() != "mesh"]
    packed = pack_lights(analytic, device=device)
    mesh = pack_mesh_lights(meshes, device=device)
    table = build_light_alias_table(environment, environment_type, packed, mesh.powers, device=device)
    return LightBuffers(packed, table, mesh.vertices, mesh.triangles, mesh.params, mesh.triangle_alias_table)


__all__ = ["LIGHT_TYPE_ENV", "LIGHT_TYPE_POINT", "LIGHT_TYPE_SPHERE", "LIGHT_TYPE_MESH", "MeshLightPack",
           "pack_lights", "pack_mesh_lights", "estimate_light_power", "environment_power",
           "build_light_alias_table", "light_buffers"]
