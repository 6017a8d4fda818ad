"""``Tracer``: the Python side of the drop-in, mirroring ``threedgptir_tracer.Tracer``.

Same constructor (``Tracer(conf)``), same ``render`` / ``build_acc`` methods, same
``_Autograd`` function (argument list, saved tensors, returned 13 outputs, gradient routing)
and the same ``LightBuffers`` / ``RenderOpts`` helpers as the reference
(threedgptir_tracer/tracer.py:40-975), with the native object swapped for
``ptir_b200.OptixTracer``. The threedgrut helpers the reference imports (the a-trous filter,
the PTIR mask post-processing, the CUDA timer) are used when threedgrut is importable; the
filter and the timer have local equivalents otherwise.
"""
from __future__ import annotations

import logging
import math
from dataclasses import dataclass
from enum import IntEnum

import torch
import torch.nn.functional as F

from .optix_tracer import OptixTracer
from .synthetic import SPP_PATTERNS

logger = logging.getLogger(__name__)


def _conf_get(node, key, default=None):
    """conf.get(key, default) for OmegaConf / dict / attribute objects."""
    if node is None:
        return default
    if hasattr(node, "get"):
        try:
            return node.get(key, default)
        except TypeError:
            pass
    return getattr(node, key, default)


class _AtrousFilter(torch.nn.Module):
    """3x3 [1 2 1] a-trous smoothing of [B,H,W,C] images (threedgrut/model/filters.py:6-69)."""

    def __init__(self, filter_type="none", iterations: int = 1):
        super().__init__()
        self.filter_type = "none" if filter_type is None else str(filter_type).lower()
        if self.filter_type not in ("none", "atrous"):
            raise ValueError(f"Unknown render.filter_type: {self.filter_type}")
        self.iterations = int(iterations)
        k = torch.tensor([[1.0, 2.0, 1.0], [2.0, 4.0, 2.0], [1.0, 2.0, 1.0]])
        self.register_buffer("kernel", (k / k.sum()).view(1, 1, 3, 3), persistent=False)

    def forward(self, x):
        if self.filter_type == "none" or self.iterations == 0:
            return x
        if x.ndim != 4:
            raise ValueError(f"Filter expects [B, H, W, C], got {tuple(x.shape)}")
        y = x.permute(0, 3, 1, 2).contiguous()
        k = self.kernel.to(device=y.device, dtype=y.dtype).repeat(y.shape[1], 1, 1, 1)
        for i in range(self.iterations):
            dl = 2 ** i
            y = F.conv2d(F.pad(y, (dl, dl, dl, dl), mode="replicate"), k, dilation=dl, groups=y.shape[1])
        return y.permute(0, 2, 3, 1).contiguous()


def _make_filter(kind):
    try:
        from threedgrut.model.filters import Filter  # type: ignore

        return Filter(kind)
    except Exception:
        return _AtrousFilter(kind)


_MASK_APPLIED_KEY = "_pbr_gt_mask_applied"
_MASKED_KEYS = ("pred_light", "pred_shadingnormal", "pred_material")


def _apply_mask(t, mask):
    """An NHWC image times the batch's foreground mask broadcast to it
    (threedgrut/model/ptir_helper.py:64-97)."""
    if t is None or mask is None or t.ndim != 4:
        return t
    m = mask.detach().to(device=t.device, dtype=t.dtype).clamp(0.0, 1.0)
    if m.ndim == 2:
        m = m[None, :, :, None]
    elif m.ndim == 3:
        m = m.unsqueeze(0) if (m.shape[-1] == 1 and m.shape[:2] == t.shape[1:3]) else m.unsqueeze(-1)
    elif m.ndim != 4:
        raise ValueError(f"GT mask must be 2D, 3D, or 4D, got {m.ndim}D")
    if m.shape[-1] != 1:
        m = m[..., :1]
    if m.shape[0] == 1 and t.shape[0] != 1:
        m = m.expand(t.shape[0], -1, -1, -1)
    if m.shape[:3] != t.shape[:3]:
        raise ValueError(f"GT mask shape {tuple(m.shape)} is not compatible with {tuple(t.shape)}")
    return t * m


def _post_processing(outputs, batch, visualize_lights):
    """Masks the light, shading-normal and material images with the batch's foreground mask
    (threedgrut/model/ptir_helper.py:100-122); threedgrut's own function when it is importable."""
    try:
        from threedgrut.model.ptir_helper import post_processing  # type: ignore
    except Exception:
        post_processing = None
    if post_processing is not None:
        return post_processing(outputs, batch, visualize_lights)
    mask = getattr(batch, "mask", None)
    if bool(outputs.get(_MASK_APPLIED_KEY, False)) or mask is None:
        return outputs
    out = dict(outputs)
    applied = False
    for k in _MASKED_KEYS:
        if outputs.get(k) is not None:
            out[k] = _apply_mask(outputs[k], mask)
            applied = True
    if applied:
        out[_MASK_APPLIED_KEY] = True
    return out


class _EventTimer:
    def __init__(self):
        self._s = torch.cuda.Event(enable_timing=True)
        self._e = torch.cuda.Event(enable_timing=True)

    def start(self):
        self._s.record()

    def end(self):
        self._e.record()

    def timing(self):
        self._e.synchronize()
        return self._s.elapsed_time(self._e)


@dataclass(frozen=True)
class LightBuffers:
    """Packed light tables handed to the tracer (threedgptir_tracer/tracer.py:40-119)."""

    lights: torch.Tensor
    alias_table: torch.Tensor
    mesh_vertices: torch.Tensor
    mesh_triangles: torch.Tensor
    mesh_lights: torch.Tensor
    mesh_triangle_alias_table: torch.Tensor

    @classmethod
    def empty(cls, device) -> "LightBuffers":
        f = dict(dtype=torch.float32, device=device)
        return cls(torch.empty((0, 9), **f), torch.empty((5, 0), **f), torch.empty((0, 3), **f),
                   torch.empty((0, 3), dtype=torch.int32, device=device), torch.empty((0, 8), **f),
                   torch.empty((3, 0), **f))

    @classmethod
    def from_batch(cls, batch, device) -> "LightBuffers":
        e = cls.empty(device)

        def pick(name, fallback):
            v = getattr(batch, name, None)
            return fallback if v is None else v

        return cls(pick("lights", e.lights), pick("light_alias_table", e.alias_table),
                   pick("mesh_light_vertices", e.mesh_vertices), pick("mesh_light_triangles", e.mesh_triangles),
                   pick("mesh_lights", e.mesh_lights),
                   pick("mesh_light_triangle_alias_table", e.mesh_triangle_alias_table)).to(device)

    def to(self, device) -> "LightBuffers":
        f = lambda t: t.to(device=device, dtype=torch.float32).contiguous()  # noqa: E731
        return LightBuffers(f(self.lights), f(self.alias_table), f(self.mesh_vertices),
                            self.mesh_triangles.to(device=device, dtype=torch.int32).contiguous(), f(self.mesh_lights),
                            f(self.mesh_triangle_alias_table))

    def tensors(self):
        return (self.lights, self.alias_table, self.mesh_vertices, self.mesh_triangles, self.mesh_lights,
                self.mesh_triangle_alias_table)


class Tracer:
    class _Autograd(torch.autograd.Function):
        """Forward = OptixTracer.trace, backward = OptixTracer.trace_bwd
        (threedgptir_tracer/tracer.py:137-384)."""

        @staticmethod
        def forward(ctx, tracer_wrapper, frame_id, ray_to_world, ray_ori, ray_dir, mog_pos, mog_rot, mog_scl, mog_dns,
                    mog_sph, mog_snrm, mog_malb, mog_mrgh, mog_mmet, environment, environment_alias_table,
                    light_buffers, render_opts, sph_degree, min_transmittance, max_bounces):
            particle_density = torch.concat([mog_pos, mog_dns, mog_rot, mog_scl, torch.zeros_like(mog_dns)], dim=1)
            particle_material = torch.concat([mog_malb, mog_mrgh, mog_mmet], dim=1)
            lights = light_buffers.to(ray_dir.device).tensors()
            out = tracer_wrapper.trace(frame_id, ray_to_world, ray_ori, ray_dir, particle_density, particle_material,
                                       mog_sph, mog_snrm, environment, environment_alias_table, *lights, render_opts,
                                       sph_degree, min_transmittance, max_bounces)
            (ray_radiance, ray_density, ray_hit_distance, ray_hit_distance_second_moment, ray_depth_distortion,
             ray_normals, ray_shadingnormal, ray_material, hits_count, mog_visibility, ray_pbr, ray_light,
             pbr_components) = out
            ctx.save_for_backward(ray_to_world, ray_ori, ray_dir, ray_radiance, ray_density, ray_hit_distance,
                                  ray_hit_distance_second_moment, ray_depth_distortion, ray_normals, ray_shadingnormal,
                                  ray_material, ray_pbr, ray_light, particle_density, particle_material, mog_sph,
                                  mog_snrm, environment, environment_alias_table, *lights)
            ctx.frame_id = frame_id
            ctx.render_opts = render_opts
            ctx.sph_degree = sph_degree
            ctx.min_transmittance = min_transmittance
            ctx.max_bounces = max_bounces
            ctx.tracer_wrapper = tracer_wrapper
            return (ray_radiance, ray_density, ray_hit_distance[:, :, :, 0:1], ray_hit_distance_second_moment,
                    ray_depth_distortion, ray_normals, ray_shadingnormal, ray_material, hits_count, mog_visibility,
                    ray_pbr, ray_light, pbr_components)

        @staticmethod
        def backward(ctx, ray_radiance_grd, ray_density_grd, ray_hit_distance_grd, ray_hit_distance_second_moment_grd,
                     ray_depth_distortion_grd, ray_normals_grd, ray_shadingnormal_grd, ray_material_grd,
                     ray_hits_count_grd_unused, mog_visibility_grd_unused, ray_pbr_grd, ray_light_grd,
                     pbr_components_grd_unused):
            (ray_to_world, ray_ori, ray_dir, ray_radiance, ray_density, ray_hit_distance, ray_hit_distance_second_moment,
             ray_depth_distortion, ray_normals, ray_shadingnormal, ray_material, ray_pbr, ray_light, particle_density,
             particle_material, mog_sph, mog_snrm, environment, environment_alias_table, *lights) = ctx.saved_tensors
            if ray_light_grd is None:
                ray_light_grd = torch.zeros_like(ray_light)

            def z(g, like):
                return torch.zeros_like(like) if g is None else g

            (particle_density_grd, particle_material_grd, mog_sph_grd, mog_sn_grd,
             environment_grd) = ctx.tracer_wrapper.trace_bwd(
                ctx.frame_id, ray_to_world, ray_ori, ray_dir, ray_radiance, ray_density, ray_hit_distance,
                ray_hit_distance_second_moment, ray_depth_distortion, ray_normals, ray_shadingnormal, ray_material,
                ray_pbr, ray_light, particle_density, particle_material, mog_sph, mog_snrm, environment,
                environment_alias_table, *lights, z(ray_radiance_grd, ray_radiance), z(ray_density_grd, ray_density),
                z(ray_hit_distance_grd, ray_hit_distance), z(ray_hit_distance_second_moment_grd,
                                                             ray_hit_distance_second_moment),
                z(ray_depth_distortion_grd, ray_depth_distortion), z(ray_normals_grd, ray_normals),
                z(ray_shadingnormal_grd, ray_shadingnormal), z(ray_material_grd, ray_material),
                z(ray_pbr_grd, ray_pbr), ray_light_grd, ctx.render_opts, ctx.sph_degree, ctx.min_transmittance,
                ctx.max_bounces)
            mog_pos_grd, mog_dns_grd, mog_rot_grd, mog_scl_grd, _ = torch.split(particle_density_grd, [3, 1, 4, 3, 1],
                                                                                dim=1)
            mog_malb_grd, mog_mrgh_grd, mog_mmet_grd = torch.split(particle_material_grd, [3, 1, 1], dim=1)
            return (None, None, None, None, None, mog_pos_grd, mog_rot_grd, mog_scl_grd, mog_dns_grd, mog_sph_grd,
                    mog_sn_grd, mog_malb_grd, mog_mrgh_grd, mog_mmet_grd, environment_grd, None, None, None, None, None,
                    None)

    class RenderOpts(IntEnum):
        NONE = 0
        INDIRECT = 1
        DEFAULT = NONE

    _MULTISPP_PATTERNS = SPP_PATTERNS

    def __init__(self, conf):
        self.device = "cuda"
        self.conf = conf
        self.num_update_bvh = 0
        self._warned_spp_fallback = False
        r = conf.render
        self.pred_pbr_filter = _make_filter(_conf_get(r, "filter_type", "none"))
        self.visualize_lights = bool(_conf_get(r, "visualize_lights", False))
        torch.zeros(1, device=self.device)  # create the CUDA context
        enable_metallic = _conf_get(r, "enable_metallic", None)
        if enable_metallic is None:
            enable_metallic = _conf_get(_conf_get(conf, "model"), "optimize_material_metallic", False)
        # B200 launch shape and attribute storage (render.b200.*; absent keys keep the defaults)
        b2 = _conf_get(r, "b200")
        launch = {k: _conf_get(b2, k) for k in ("schedule", "chunk_tiles", "kbuffer", "refill_lanes", "block_size",
                                                 "sort_rays", "storage", "shadow_kbuffer", "exact_candidates",
                                                 "resume_rounds", "bvh_builder")}
        self.tracer_wrapper = OptixTracer(
            "", "", r.pipeline_type, r.backward_pipeline_type, r.primitive_type, r.particle_kernel_degree,
            r.particle_kernel_min_response, r.particle_kernel_density_clamping, r.particle_radiance_sph_degree,
            r.enable_normals, r.enable_hitcounts, r.enable_mis, bool(enable_metallic), self.visualize_lights,
            **{k: v for k, v in launch.items() if v is not None})
        self.frame_timer = _EventTimer() if _conf_get(r, "enable_kernel_timings", False) else None
        self.timings = {}

    # ---- output bookkeeping (threedgptir_tracer/tracer.py:471-536)
    def _required_train_output_keys(self):
        keys = {"pred_pbr", "pred_material"}
        loss = _conf_get(self.conf, "loss")
        if bool(_conf_get(loss, "use_light_consistency", False)) or float(_conf_get(loss, "lambda_light", 0.0)) > 0.0:
            keys.add("pred_light")
        if bool(_conf_get(loss, "use_edge_aware_smoothness", False)):
            keys.update(_conf_get(loss, "edge_aware_smoothness_outputs", []))
        return keys

    def _train_output_key_sets(self, train):
        if not train or not bool(_conf_get(self.conf.render, "hide_intermediate_outputs", False)):
            return None, None
        final = self._required_train_output_keys()
        acc = set(final)
        if "pred_pbr" in acc:
            acc.add("pred_opacity")
        if "pred_direct" in acc or "pred_indirect" in acc:
            acc.update(("pbr_components", "pred_opacity"))
        return final, acc

    def _postprocess_pbr_outputs(self, outputs):
        op = outputs.get("pred_opacity")
        keys = ("pred_pbr", "pred_direct", "pred_indirect")
        if op is not None:
            for k in keys:
                if outputs.get(k) is not None:
                    outputs[k] = outputs[k] * op
        for k in (*keys, "pred_light"):
            if outputs.get(k) is not None:
                outputs[k] = self.pred_pbr_filter(outputs[k])

    @staticmethod
    def _normalize_depth_output(outputs):
        d, op = outputs.get("pred_dist"), outputs.get("pred_opacity")
        if d is not None and op is not None:
            outputs["pred_dist"] = torch.nan_to_num(d / op, 0.0, 0.0)

    def _get_spp(self, train):
        return max(1, int(self.conf.render.inversion_spp if train else self.conf.render.render_spp))

    def _get_spp_chunk(self, spp):
        return min(spp, max(1, int(_conf_get(self.conf.render, "spp_chunk", spp))))

    def _warn_spp_fallback(self, reason):
        if not self._warned_spp_fallback:
            logger.warning("PTIR SPP fallback to spp=1: %s.", reason)
            self._warned_spp_fallback = True

    # ---- sample expansion (threedgptir_tracer/tracer.py:537-706)
    @staticmethod
    def _flat(value, dtype, device):
        return None if value is None else torch.as_tensor(value, dtype=dtype, device=device).flatten()

    def _extract_pinhole_intrinsics(self, batch, dtype, device, warn=True):
        intr = self._flat(getattr(batch, "intrinsics", None), dtype, device)
        if intr is not None:
            if intr.numel() == 4:
                return tuple(intr)
            if intr.numel() == 9:
                K = intr.reshape(3, 3)
                return K[0, 0], K[1, 1], K[0, 2], K[1, 2]
            if warn:
                self._warn_spp_fallback("unsupported intrinsics format")
            return None
        params = getattr(batch, "intrinsics_OpenCVPinholeCameraModelParameters", None)
        if params is None:
            if warn:
                self._warn_spp_fallback("missing pinhole intrinsics")
            return None

        def get(name):
            return params.get(name) if isinstance(params, dict) else getattr(params, name, None)

        for name in ("radial_coeffs", "tangential_coeffs", "thin_prism_coeffs"):
            c = self._flat(get(name), dtype, device)
            if c is not None and c.numel() > 0 and torch.any(torch.abs(c) > 1e-8).item():
                if warn:
                    self._warn_spp_fallback("distorted camera model")
                return None
        focal = self._flat(get("focal_length"), dtype, device)
        principal = self._flat(get("principal_point"), dtype, device)
        if focal is None or principal is None or focal.numel() < 1 or principal.numel() < 2:
            if warn:
                self._warn_spp_fallback("incomplete pinhole intrinsics")
            return None
        fx = focal[0]
        fy = focal[1] if focal.numel() > 1 else focal[0]
        return fx, fy, principal[0], principal[1]

    def _can_expand_spp(self, batch):
        return getattr(batch, "pixel_coords", None) is not None and self._extract_pinhole_intrinsics(
            batch, batch.rays_dir.dtype, batch.rays_dir.device, warn=False) is not None

    def _make_spp_jitter(self, spp, h, w, device, dtype, frame_id):
        if spp in self._MULTISPP_PATTERNS:
            return torch.tensor(self._MULTISPP_PATTERNS[spp], dtype=dtype, device=device).view(spp, 1, 1, 2)
        gw = int(math.ceil(math.sqrt(spp)))
        gh = int(math.ceil(spp / gw))
        idx = torch.arange(spp, dtype=dtype, device=device)
        jitter = torch.stack(((torch.remainder(idx, gw) + 0.5) / gw,
                              (torch.div(idx, gw, rounding_mode="floor") + 0.5) / gh), dim=-1)
        gen = torch.Generator(device=device)
        gen.manual_seed((int(frame_id) + 1) * 1315423911 + spp * 2654435761)
        shift = torch.rand((1, 2), dtype=dtype, device=device, generator=gen)
        return torch.remainder(jitter + shift, 1.0).view(spp, 1, 1, 2)

    def _expand_rays_for_spp(self, batch, spp, frame_id, jitter=None):
        rays_ori = batch.rays_ori.contiguous()
        rays_dir = batch.rays_dir.contiguous()
        if spp == 1 and jitter is None:
            return rays_ori, rays_dir, 1
        pixel_coords = getattr(batch, "pixel_coords", None)
        intr = self._extract_pinhole_intrinsics(batch, rays_dir.dtype, rays_dir.device)
        if intr is None or pixel_coords is None:
            if pixel_coords is None:
                self._warn_spp_fallback("batch has no pixel_coords")
            return rays_ori, rays_dir, 1
        base, h, w, _ = rays_dir.shape
        fx, fy, cx, cy = intr
        origin = (pixel_coords.to(dtype=rays_dir.dtype, device=rays_dir.device) - 0.5).unsqueeze(0)
        if jitter is None:
            jitter = self._make_spp_jitter(spp, h, w, rays_dir.device, rays_dir.dtype, frame_id)
        jitter = jitter.view(spp, 1, 1, 1, 2) if jitter.shape[1:3] == (1, 1) else jitter.view(spp, 1, h, w, 2)
        dirs = torch.stack(((origin[..., 0] + jitter[..., 0] - cx) / fx, (origin[..., 1] + jitter[..., 1] - cy) / fy,
                            torch.ones((spp, base, h, w), dtype=rays_dir.dtype, device=rays_dir.device)), dim=-1)
        dirs = F.normalize(dirs, dim=-1).reshape(spp * base, h, w, 3).contiguous()
        origins = rays_ori.unsqueeze(0).expand(spp, *rays_ori.shape).reshape(spp * base, h, w, 3).contiguous()
        return origins, dirs, spp

    @staticmethod
    def _average_spp_output(value, spp, base):
        return value if spp == 1 else value.reshape(spp, base, *value.shape[1:]).mean(dim=0)

    # ---- acceleration structure (threedgptir_tracer/tracer.py:716-738)
    def build_acc(self, gaussians, rebuild=True):
        r = self.conf.render
        allow_update = (r.max_consecutive_bvh_update > 1) and not r.particle_kernel_density_clamping
        rebuild_bvh = rebuild or r.particle_kernel_density_clamping or self.num_update_bvh >= r.max_consecutive_bvh_update
        self.tracer_wrapper.build_bvh(
            gaussians.positions.view(-1, 3).contiguous(),
            gaussians.rotation_activation(gaussians.rotation).view(-1, 4).contiguous(),
            gaussians.scale_activation(gaussians.scale).view(-1, 3).contiguous(),
            gaussians.density_activation(gaussians.density).view(-1, 1).contiguous(), rebuild_bvh, allow_update)
        self.num_update_bvh = 0 if rebuild_bvh else self.num_update_bvh + 1

    # ---- render (threedgptir_tracer/tracer.py:740-975)
    def render(self, gaussians, gpu_batch, train=False, frame_id=0, sh_indirect: bool = False):
        if self.frame_timer is not None:
            self.frame_timer.start()
        base = gpu_batch.rays_dir.shape[0]
        spp = self._get_spp(train)
        if spp > 1 and not self._can_expand_spp(gpu_batch):
            self._warn_spp_fallback("batch has no supported pinhole intrinsics/pixel_coords")
            spp = 1
        chunk = self._get_spp_chunk(spp)
        h, w = gpu_batch.rays_dir.shape[1:3]
        jitter = None
        if spp > 1:
            jitter = self._make_spp_jitter(spp, h, w, gpu_batch.rays_dir.device, gpu_batch.rays_dir.dtype, frame_id)
        final_keys, acc_keys = self._train_output_key_sets(train)
        acc = {}
        mog_visibility = None
        total_spp = 0
        for start in range(0, spp, chunk):
            n_spp = min(chunk, spp - start)
            cj = None if jitter is None else jitter[start:start + n_spp]
            rays_ori, rays_dir, n_spp = self._expand_rays_for_spp(gpu_batch, n_spp, frame_id + start, jitter=cj)
            environment = gaussians.get_environment()
            if environment is None:
                environment = torch.empty((0, 0, 4), dtype=torch.float32, device=rays_dir.device)
            alias = getattr(gaussians, "environment_alias_table", None)
            if alias is None:
                alias_t = torch.empty(0, dtype=torch.float32, device=rays_dir.device)
            else:
                alias_t = torch.concat([alias.prob.reshape(1, alias.height, alias.width),
                                        alias.alias.reshape(1, alias.height, alias.width).to(dtype=torch.float32),
                                        alias.pdf.reshape(1, alias.height, alias.width)], dim=0).to(
                    device=rays_dir.device).contiguous()
            lights = LightBuffers.from_batch(gpu_batch, device=rays_dir.device)
            out = Tracer._Autograd.apply(
                self.tracer_wrapper, frame_id + start, gpu_batch.T_to_world.contiguous(), rays_ori, rays_dir,
                gaussians.positions.contiguous(), gaussians.get_rotation().contiguous(),
                gaussians.get_scale().contiguous(), gaussians.get_density().contiguous(),
                gaussians.get_features().contiguous(), gaussians.get_shading_normal().contiguous(),
                gaussians.get_material_albedo().contiguous(), gaussians.get_material_roughness().contiguous(),
                gaussians.get_material_metallic().contiguous(), environment, alias_t, lights,
                int(Tracer.RenderOpts.INDIRECT if sh_indirect else Tracer.RenderOpts.DEFAULT),
                gaussians.n_active_features, self.conf.render.min_transmittance,
                _conf_get(self.conf.render, "max_bounces", 3))
            (rgb, opacity, dist, dist2, distortion, normals, snormal, material, hits, vis, pbr, light, comps) = out
            rgb, opacity = gaussians.background(gpu_batch.T_to_world.contiguous(), rays_dir, rgb, opacity, train)
            for name, value in (("pred_rgb", rgb), ("pred_opacity", opacity), ("pred_dist", dist),
                                ("pred_depth_second_moment", dist2), ("pred_depth_distortion", distortion),
                                ("pred_normals", normals), ("pred_shadingnormal", snormal), ("pred_material", material),
                                ("hits_count", hits), ("pred_pbr", pbr), ("pred_light", light),
                                ("pbr_components", comps.detach())):
                if acc_keys is not None and name not in acc_keys:
                    continue
                weighted = self._average_spp_output(value, n_spp, base) * n_spp
                acc[name] = weighted if name not in acc else acc[name] + weighted
            mog_visibility = vis if mog_visibility is None else torch.maximum(mog_visibility, vis)
            total_spp += n_spp
        if self.frame_timer is not None:
            self.frame_timer.end()
        acc = {k: v / total_spp for k, v in acc.items()}
        comps = acc.pop("pbr_components", None)
        if comps is not None:
            acc["pred_direct"] = comps[..., 0, :]
            acc["pred_indirect"] = comps[..., 1, :]
        self._normalize_depth_output(acc)
        self._postprocess_pbr_outputs(acc)
        if self.frame_timer is not None:
            self.timings["forward_render"] = self.frame_timer.timing()
        keys = ("pred_rgb", "pred_opacity", "pred_dist", "pred_depth_second_moment", "pred_depth_distortion",
                "pred_normals", "pred_shadingnormal", "pred_material", "pred_pbr", "pred_light", "pred_direct",
                "pred_indirect", "hits_count")
        vals = {k: acc.get(k) for k in keys}
        if vals["pred_normals"] is not None:
            vals["pred_normals"] = F.normalize(vals["pred_normals"], dim=3)
        outputs = {k: v for k, v in vals.items() if v is not None and (final_keys is None or k in final_keys)}
        outputs["frame_time_ms"] = self.frame_timer.timing() if self.frame_timer is not None else 0.0
        outputs["mog_visibility"] = mog_visibility
        return _post_processing(outputs, gpu_batch, self.visualize_lights)
