"""Seeded synthetic scenes, cameras and environments of the benchmark workloads.

Every workload is a Gaussian field plus pinhole views plus an equirect environment, generated
from one integer seed with numpy's PCG64 so that tests, the benchmark and the oracle see the
same bytes. The five workloads:

  field-10k      10,000 Gaussians, 1 view 128x128, 1 spp, 2 bounces, env 64x128, forward only
  field-100k     100,000 Gaussians, 1 view 400x400, 4 spp, 3 bounces, env 256x512, fwd+bwd
  field-300k-mv  300,000 Gaussians, 16 views of {256,400,512,800}^2 with spp in {1,2,4,8,16}
  field-300k-sh  300,000 Gaussians with degree-3 SH ~ N(0,0.1), 800x800, 8 spp, 3 bounces
  field-1m       1,000,000 Gaussians (70% N(0,I) cluster, 30% shell of radius U[5,20]),
                 8 views 1024x768, 16 spp, 4 bounces, env 512x1024, fwd+bwd
Gaussians: means U[-1,1]^3 (except field-1m), per-axis scales log-uniform, rotations uniform
unit quaternions (wxyz), opacity sigmoid(N(0,1)), albedo U[0,1]^3, roughness U[0.05,1],
metallic U[0,1], shading normals uniform unit vectors, SH DC ~ N(0,0.5) and higher orders 0
unless stated. Environment RGB ~ LogNormal(0,1), alpha 1. Views sit uniformly on the sphere of
radius 3 looking at the origin, 40 degree vertical field of view.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

# sub-pixel sample offsets per pixel for the standard sample counts (the same table as the
# reference's Tracer._MULTISPP_PATTERNS, threedgptir_tracer/tracer.py:391-426)
SPP_PATTERNS = {
    1: ((0.5, 0.5),),
    2: ((0.25, 0.25), (0.75, 0.75)),
    4: ((0.375, 0.125), (0.875, 0.375), (0.625, 0.875), (0.125, 0.625)),
    8: ((0.5625, 0.6875), (0.4375, 0.3125), (0.8125, 0.4375), (0.3125, 0.8125), (0.1875, 0.1875),
        (0.0625, 0.5625), (0.6875, 0.0625), (0.9375, 0.9375)),
    16: ((0.5625, 0.4375), (0.4375, 0.6875), (0.3125, 0.375), (0.75, 0.5625), (0.1875, 0.625), (0.625, 0.1875),
         (0.1875, 0.3125), (0.6875, 0.8125), (0.375, 0.125), (0.5, 0.9375), (0.25, 0.875), (0.125, 0.25),
         (0.0, 0.5), (0.9375, 0.75), (0.875, 0.0625), (0.0625, 0.0)),
    32: tuple(((x + 0.5) / 8.0, (y + 0.5) / 4.0) for y in range(4) for x in range(8)),
}


@dataclass
class Workload:
    name: str
    n: int
    views: list  # [(width, height, spp)]
    max_bounces: int
    env_hw: tuple
    layout: str = "uniform"         # "uniform" | "cluster_shell"
    scale_range: tuple = (0.005, 0.05)
    sh_full: bool = False
    backward: bool = True
    seed: int = 0
    extra: dict = field(default_factory=dict)


def workload(name: str, seed: int = 0) -> Workload:
    if name == "field-10k":
        return Workload(name, 10_000, [(128, 128, 1)], 2, (64, 128), backward=False, seed=seed)
    if name == "field-100k":
        return Workload(name, 100_000, [(400, 400, 4)], 3, (256, 512), seed=seed)
    if name == "field-300k-mv":
        rng = np.random.default_rng(seed + 7)
        views = [(int(r), int(r), int(s)) for r, s in zip(rng.choice([256, 400, 512, 800], 16), rng.choice([1, 2, 4, 8, 16], 16))]
        return Workload(name, 300_000, views, 3, (512, 1024), seed=seed)
    if name == "field-300k-sh":
        return Workload(name, 300_000, [(800, 800, 8)], 3, (512, 1024), sh_full=True, seed=seed)
    if name == "field-1m":
        return Workload(name, 1_000_000, [(1024, 768, 16)] * 8, 4, (512, 1024), layout="cluster_shell",
                        scale_range=(0.002, 0.2), seed=seed)
    raise KeyError(name)


def _unit(rng, n, d):
    v = rng.standard_normal((n, d))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


def make_field(n: int, seed: int = 0, layout: str = "uniform", scale_range=(0.005, 0.05), sh_degree: int = 3,
               sh_full: bool = False) -> dict:
    """Gaussian field as float32 CPU tensors: pos [n,3], rot [n,4] (wxyz), scl [n,3], dns [n,1],
    albedo [n,3], roughness [n,1], metallic [n,1], snrm [n,3], sph [n,(d+1)^2*3]."""
    rng = np.random.default_rng(seed)
    if layout == "uniform":
        pos = rng.uniform(-1.0, 1.0, (n, 3))
    elif layout == "cluster_shell":
        nc = int(round(0.7 * n))
        core = rng.standard_normal((nc, 3))
        shell = _unit(rng, n - nc, 3) * rng.uniform(5.0, 20.0, (n - nc, 1))
        pos = np.concatenate([core, shell], 0)
    else:
        raise ValueError(layout)
    lo, hi = math.log(scale_range[0]), math.log(scale_range[1])
    scl = np.exp(rng.uniform(lo, hi, (n, 3)))
    rot = _unit(rng, n, 4)
    dns = 1.0 / (1.0 + np.exp(-rng.standard_normal((n, 1))))
    albedo = rng.uniform(0.0, 1.0, (n, 3))
    rough = rng.uniform(0.05, 1.0, (n, 1))
    metal = rng.uniform(0.0, 1.0, (n, 1))
    snrm = _unit(rng, n, 3)
    nc = (sh_degree + 1) ** 2
    sph = np.zeros((n, nc * 3))
    if sh_full:
        sph[:] = rng.normal(0.0, 0.1, (n, nc * 3))
    else:
        sph[:, :3] = rng.normal(0.0, 0.5, (n, 3))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32))  # noqa: E731
    return dict(pos=t(pos), rot=t(rot), scl=t(scl), dns=t(dns), albedo=t(albedo), roughness=t(rough),
                metallic=t(metal), snrm=t(snrm), sph=t(sph))


def make_environment(h: int, w: int, seed: int = 0) -> torch.Tensor:
    rng = np.random.default_rng(seed + 1)
    env = np.ones((h, w, 4), np.float32)
    env[..., :3] = rng.lognormal(0.0, 1.0, (h, w, 3))
    return torch.from_numpy(env)


def camera_positions(count: int, seed: int = 0, radius: float = 3.0) -> np.ndarray:
    rng = np.random.default_rng(seed + 2)
    return _unit(rng, count, 3) * radius


def pinhole_rays(width: int, height: int, eye, fov_deg: float = 40.0, jitter=(0.5, 0.5), look_at=(0.0, 0.0, 0.0)):
    """World-space rays of a pinhole camera: (origins [h,w,3], unit directions [h,w,3]) float32."""
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(look_at, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    up = np.array([0.0, 0.0, 1.0])
    if abs(np.dot(up, fwd)) > 0.999:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    th = math.tan(math.radians(fov_deg) * 0.5)
    tw = th * width / height
    xs = (np.arange(width) + jitter[0]) / width * 2.0 - 1.0
    ys = 1.0 - (np.arange(height) + jitter[1]) / height * 2.0
    X, Y = np.meshgrid(xs, ys)
    d = fwd[None, None, :] + X[..., None] * tw * right[None, None, :] + Y[..., None] * th * upv[None, None, :]
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    o = np.broadcast_to(eye, d.shape)
    return np.ascontiguousarray(o, np.float32), np.ascontiguousarray(d, np.float32)


def view_rays(width: int, height: int, spp: int, eye, fov_deg: float = 40.0):
    """Rays of all samples of one view, [spp, h, w, 3] each (sample offsets from SPP_PATTERNS,
    or a stratified grid for other counts)."""
    pattern = SPP_PATTERNS.get(spp)
    if pattern is None:
        gw = int(math.ceil(math.sqrt(spp)))
        gh = int(math.ceil(spp / gw))
        pattern = tuple((((i % gw) + 0.5) / gw, ((i // gw) + 0.5) / gh) for i in range(spp))
    os_, ds = [], []
    for j in pattern:
        o, d = pinhole_rays(width, height, eye, fov_deg, j)
        os_.append(o)
        ds.append(d)
    return torch.from_numpy(np.stack(os_)), torch.from_numpy(np.stack(ds))


def view_rays_device(width: int, height: int, spp: int, eye, device, fov_deg: float = 40.0):
    """Same rays as view_rays(), computed with torch on `device` (float32): [spp, h, w, 3] x 2."""
    pattern = SPP_PATTERNS.get(spp)
    if pattern is None:
        gw = int(math.ceil(math.sqrt(spp)))
        gh = int(math.ceil(spp / gw))
        pattern = tuple((((i % gw) + 0.5) / gw, ((i // gw) + 0.5) / gh) for i in range(spp))
    eye = np.asarray(eye, np.float64)
    fwd = -eye / np.linalg.norm(eye)
    up = np.array([0.0, 0.0, 1.0])
    if abs(np.dot(up, fwd)) > 0.999:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    th = math.tan(math.radians(fov_deg) * 0.5)
    tw = th * width / height
    f64 = dict(dtype=torch.float64, device=device)
    jit = torch.tensor(pattern, **f64)  # [spp, 2]
    xs = (torch.arange(width, **f64)[None, :] + jit[:, :1]) / width * 2.0 - 1.0  # [spp, w]
    ys = 1.0 - (torch.arange(height, **f64)[None, :] + jit[:, 1:]) / height * 2.0  # [spp, h]
    F, Rt, U = (torch.tensor(v, **f64) for v in (fwd, right, upv))
    d = (F[None, None, None, :] + xs[:, None, :, None] * tw * Rt + ys[:, :, None, None] * th * U)
    d = d / torch.linalg.norm(d, dim=-1, keepdim=True)
    o = torch.tensor(eye, **f64).expand_as(d)
    return o.float().contiguous(), d.float().contiguous()


def density_tensor(f: dict) -> torch.Tensor:
    """[n,12] = pos, density, rot (wxyz), scale, 0 (threedgptir_tracer/tracer.py:163-165)."""
    return torch.cat([f["pos"], f["dns"], f["rot"], f["scl"], torch.zeros_like(f["dns"])], 1).contiguous()


def material_tensor(f: dict) -> torch.Tensor:
    """[n,5] = albedo, roughness, metallic (threedgptir_tracer/tracer.py:166)."""
    return torch.cat([f["albedo"], f["roughness"], f["metallic"]], 1).contiguous()
