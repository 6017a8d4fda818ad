"""Environment-map importance table (the input producer of the tracer's NEE).

Same table as the reference's ``build_environment_alias_table``
(threedgrut/model/aliastable.py:244-297): the map is area-resized to 64x128 (equirect), weighted
by Rec.709 luminance times texel solid angle, and turned into a Walker/Vose alias table whose
construction order (index-ordered small/large stacks, pop from the end) is kept so that the
table is identical; the pdf is per steradian. ``pack`` gives the [3, h, w] float tensor the
tracer reads (threedgptir_tracer/tracer.py:824-847).
"""
from __future__ import annotations

import math

import numpy as np
import torch
import torch.nn.functional as F

ALIAS_TABLE_SIZE = (64, 128)
LUMINANCE = (0.2126, 0.7152, 0.0722)


def vose(weights: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Alias table (prob float32, alias int64) of non-negative weights, built in float64."""
    w = np.asarray(weights, dtype=np.float64).reshape(-1)
    w = np.where(np.isfinite(w) & (w > 0.0), w, 0.0)
    n = w.size
    total = float(w.sum())
    alias = np.arange(n, dtype=np.int64)
    prob = np.ones(n, dtype=np.float32)
    if total <= 0.0:
        return prob, alias
    scaled = w * (float(n) / total)
    small = [int(i) for i in np.nonzero(scaled < 1.0)[0]]
    large = [int(i) for i in np.nonzero(scaled >= 1.0)[0]]
    while small and large:
        s = small.pop()
        g = large.pop()
        prob[s] = np.float32(min(max(scaled[s], 0.0), 1.0))
        alias[s] = g
        scaled[g] -= 1.0 - scaled[s]
        (small if scaled[g] < 1.0 else large).append(g)
    for i in small + large:
        prob[i] = 1.0
        alias[i] = i
    return prob, alias


def _solid_angles_equirect(h: int, w: int) -> torch.Tensor:
    edges = (torch.arange(h + 1, dtype=torch.float32) / float(h) - 0.5) * math.pi
    rows = (2.0 * math.pi / float(w)) * (torch.sin(edges[1:]) - torch.sin(edges[:-1]))
    return torch.clamp(rows, min=0.0).reshape(h, 1).expand(h, w).contiguous()


def _solid_angles_cube(fs: int) -> torch.Tensor:
    e = torch.linspace(-1.0, 1.0, fs + 1, dtype=torch.float32)
    u0, u1 = e[:-1].reshape(1, fs), e[1:].reshape(1, fs)
    v0, v1 = e[:-1].reshape(fs, 1), e[1:].reshape(fs, 1)

    def area(u, v):
        return torch.atan2(u * v, torch.sqrt(u * u + v * v + 1.0))

    sa = area(u1, v1) - area(u0, v1) - area(u1, v0) + area(u0, v0)
    return torch.clamp(sa, min=0.0).repeat(6, 1).contiguous()


def build(environment: torch.Tensor, cube: bool | None = None, size=ALIAS_TABLE_SIZE) -> dict:
    """Alias table of an [H, W, C>=3] environment (CPU computation). Returns dict with
    width, height, prob [h*w] f32, alias [h*w] i32, pdf [h*w] f32."""
    env = environment.detach().to("cpu", torch.float32)
    H, W = env.shape[:2]
    if cube is None:
        cube = H == 6 * W
    if not cube and size is not None and tuple(env.shape[:2]) != tuple(size):
        env = F.interpolate(env.permute(2, 0, 1).unsqueeze(0), size=tuple(size), mode="area").squeeze(0).permute(1, 2, 0)
    rgb = env[..., :3]
    rgb = torch.where(torch.isfinite(rgb) & (rgb > 0.0), rgb, torch.zeros_like(rgb))
    lum = torch.sum(rgb * rgb.new_tensor(LUMINANCE), dim=-1)
    h, w = lum.shape
    sa = _solid_angles_cube(w) if cube else _solid_angles_equirect(h, w)
    weights = (lum * sa).contiguous()
    total = weights.sum()
    if not bool(torch.isfinite(total)) or float(total) <= 0.0:
        weights = sa
        total = weights.sum()
    pdf = torch.where(sa > 0.0, weights / torch.clamp(total * sa, min=torch.finfo(torch.float32).tiny), torch.zeros_like(weights))
    prob, alias = vose(weights.numpy())
    return dict(width=int(w), height=int(h), prob=torch.from_numpy(prob), alias=torch.from_numpy(alias.astype(np.int32)),
                pdf=pdf.reshape(-1).contiguous())


def build_device(environment: torch.Tensor, size=ALIAS_TABLE_SIZE) -> torch.Tensor:
    """The packed [3, h, w] table of build() + pack(), computed on the environment's CUDA device
    by the library (ptir_build_env_table): same algorithm and Vose order, float64 on the device."""
    from . import _native as N

    env = environment.detach()
    if env.dtype != torch.float32 or not env.is_cuda or env.dim() != 3 or env.shape[2] < 3:
        raise ValueError("build_device: a [H, W, C>=3] float32 CUDA tensor is required")
    env = env.contiguous()
    H, W, Ch = (int(v) for v in env.shape)
    h, w = (H, W) if H == 6 * W else (int(size[0]), int(size[1]))
    lib = N.load()
    scratch = torch.empty(int(lib.ptir_env_table_scratch_bytes(h * w)), dtype=torch.uint8, device=env.device)
    out = torch.empty((3, h, w), dtype=torch.float32, device=env.device)
    rc = lib.ptir_build_env_table(env.data_ptr(), H, W, Ch, h, w, out.data_ptr(), scratch.data_ptr(),
                                  scratch.numel(), torch.cuda.current_stream(env.device).cuda_stream)
    if rc != N.PTIR_OK:
        raise N.PtirError(rc, "ptir_build_env_table failed")
    return out


def pack(table: dict, device=None) -> torch.Tensor:
    """[3, h, w] float32: prob, alias index as float, pdf."""
    h, w = table["height"], table["width"]
    t = torch.stack([table["prob"].reshape(h, w).float(), table["alias"].reshape(h, w).float(),
                     table["pdf"].reshape(h, w).float()], dim=0).contiguous()
    return t if device is None else t.to(device)
