"""Host-side render fixtures shared by tests/golden/make_render_golden.py and
tests/test_render_host.py.

``Tracer.render`` / ``Tracer._Autograd`` / ``Tracer.build_acc`` (threedgptir_tracer/tracer.py:137-975)
turn a batch and a Gaussian model into plugin calls (SPP jitter and ray expansion, chunking,
parameter packing, frame ids) and turn the plugin's outputs back into images (background,
SPP averaging, depth normalisation, opacity weighting, filter, mask) and its gradients into
parameter gradients (the [3,1,4,3,1] / [3,1,1] splits). To pin that host logic to the reference's
own tracer.py, both tracers run here against the same stand-in plugin, ``RecordingPlugin``: a
deterministic float32 function of every argument it is given, on the CPU, that records each
call. The golden file holds the reference's calls, images and gradients; ours must equal them
bit for bit.
"""
from __future__ import annotations

from contextlib import contextmanager

import torch
import torch.nn.functional as F


class AttrDict(dict):
    """conf node with both attribute access and .get, like the OmegaConf nodes the tracers read."""

    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError as e:
            raise AttributeError(k) from e


def _sum_or0(t):
    return t.float().sum() if isinstance(t, torch.Tensor) and t.numel() > 0 else torch.zeros(())


class RecordingPlugin:
    """Stand-in for the native ``OptixTracer``: records every call, answers deterministically."""

    def __init__(self, *args, **kwargs):
        self.ctor = args
        self.calls = []

    # buildBVH(pos, rot, scl, dns, rebuild, allow_update)
    def build_bvh(self, pos, rot, scl, dns, rebuild, allow_update=True):
        self.calls.append(("build_bvh", [pos.clone(), rot.clone(), scl.clone(), dns.clone()],
                           [int(bool(rebuild)), int(bool(allow_update))]))

    def trace(self, frame, t2w, ori, dirs, dens, mat, sph, snrm, env, alias, lights, light_alias, mesh_v, mesh_t,
              mesh_l, mesh_a, render_opts, sph_degree, min_t, max_bounces):
        tensors = [t2w, ori, dirs, dens, mat, sph, snrm, env, alias, lights, light_alias, mesh_v, mesh_t, mesh_l, mesh_a]
        self.calls.append(("trace", [t.detach().clone() for t in tensors],
                           [int(frame), int(render_opts), int(sph_degree), float(min_t), int(max_bounces)]))
        c = dens.sum(0)
        m = mat.sum(0)
        aux = (_sum_or0(env) * 1e-3 + _sum_or0(alias) * 1e-4 + _sum_or0(lights) * 1e-3 + _sum_or0(light_alias) * 1e-4
               + _sum_or0(mesh_v) * 1e-3 + _sum_or0(mesh_t) * 1e-5 + _sum_or0(mesh_l) * 1e-3 + _sum_or0(mesh_a) * 1e-4
               + sph.sum() * 1e-3 + snrm.sum() * 1e-3 + t2w.sum() * 1e-2)
        base = dirs * (1.0 + 0.01 * int(frame)) + ori * 0.1
        scal = (int(render_opts) * 0.1 + int(sph_degree) * 0.01 + float(min_t) + int(max_bounces) * 0.001)
        rad = torch.sin(base + c[0:3] * 0.01) + aux
        dns = torch.sigmoid(base.sum(-1, keepdim=True) + c[3] * 0.01)
        hit = torch.cat([base.abs().sum(-1, keepdim=True) + c[4] * 0.01, (base * base).sum(-1, keepdim=True)], -1)
        hit2 = hit[..., 1:2] * 0.5 + c[5] * 0.01
        dist = (base[..., 0:1] - base[..., 1:2]).abs() + c[6] * 0.01
        nrm = torch.cos(base * 1.3 + c[7:10] * 0.01)
        snrm_i = torch.sin(base * 0.7 + c[9:12] * 0.01)
        mat_i = torch.cos(base[..., 0:1] * (m + 1.0))
        hits = torch.floor(base.sum(-1, keepdim=True).abs() * 3.0)
        vis = torch.sigmoid(dens[:, 3:4] + int(frame) * 0.001)
        pbr = rad * (m[0:3].mean() * 0.01 + 1.0) + scal
        light = torch.cos(base + scal)
        comps = torch.stack([pbr * 0.625, pbr * 0.375], dim=-2)
        return rad, dns, hit, hit2, dist, nrm, snrm_i, mat_i, hits, vis, pbr, light, comps

    def trace_bwd(self, frame, t2w, ori, dirs, rad, dns, hit, hit2, dist, nrm, snrm_i, mat_i, pbr, light, dens, mat,
                  sph, snrm, env, alias, lights, light_alias, mesh_v, mesh_t, mesh_l, mesh_a, rad_g, dns_g, hit_g,
                  hit2_g, dist_g, nrm_g, snrm_g, mat_g, pbr_g, light_g, render_opts, sph_degree, min_t, max_bounces):
        grads = [rad_g, dns_g, hit_g, hit2_g, dist_g, nrm_g, snrm_g, mat_g, pbr_g, light_g]
        self.calls.append(("trace_bwd", [t.detach().clone() for t in grads],
                           [int(frame), int(render_opts), int(sph_degree), float(min_t), int(max_bounces)]))
        # one scalar per incoming gradient, each weighted by a saved output it belongs with
        w = torch.stack([(rad_g * rad).sum(), (dns_g * dns).sum(), (hit_g * hit[..., 0:1]).sum(), (hit2_g * hit2).sum(),
                         (dist_g * dist).sum(), (nrm_g * nrm).sum(), (snrm_g * snrm_i).sum(), (mat_g * mat_i).sum(),
                         (pbr_g * pbr).sum(), (light_g * light).sum(), (pbr_g * dirs).sum(), (rad_g * ori).sum()])
        n = dens.shape[0]
        ramp = torch.arange(1, n + 1, dtype=torch.float32).unsqueeze(1) / n
        dens_grad = ramp * w.unsqueeze(0) + dens * 0.001 * int(frame + 1)
        mat_grad = ramp * w[0:5].flip(0).unsqueeze(0) + mat * 0.01
        sph_grad = torch.cos(sph + w[8]) * ramp
        snrm_grad = snrm * w[6] + ramp * w[7]
        env_grad = (torch.sin(env + w[9]) * 0.5 if env.numel() > 0 else torch.zeros_like(env))
        return dens_grad, mat_grad, sph_grad, snrm_grad, env_grad


class AliasTable:
    def __init__(self, h, w, g):
        self.height, self.width = h, w
        self.prob = torch.rand(h * w, generator=g)
        self.alias = torch.randint(0, h * w, (h * w,), generator=g)
        self.pdf = torch.rand(h * w, generator=g)


class Gaussians:
    """The parts of threedgrut's MixtureOfGaussians that the tracer reads (activations included)."""

    def __init__(self, n=37, sph_degree=1, seed=0, environment=True, alias=True):
        g = torch.Generator().manual_seed(seed)
        p = lambda *s: torch.nn.Parameter(torch.randn(*s, generator=g))  # noqa: E731
        self.num_gaussians = n
        self.positions, self.rotation, self.scale, self.density = p(n, 3), p(n, 4), p(n, 3), p(n, 1)
        self.features = p(n, (sph_degree + 1) ** 2 * 3)
        self.shading_normal = p(n, 3)
        self.albedo, self.roughness, self.metallic = p(n, 3), p(n, 1), p(n, 1)
        self.environment = p(8, 16, 4) if environment else None
        self.environment_alias_table = AliasTable(4, 8, g) if alias else None
        self.n_active_features = sph_degree
        self.bg = torch.rand(3, generator=g)

    rotation_activation = staticmethod(lambda r: F.normalize(r, dim=-1))
    scale_activation = staticmethod(torch.exp)
    density_activation = staticmethod(torch.sigmoid)

    def params(self):
        ps = [self.positions, self.rotation, self.scale, self.density, self.features, self.shading_normal, self.albedo,
              self.roughness, self.metallic]
        return ps + ([self.environment] if self.environment is not None else [])

    def get_rotation(self):
        return self.rotation_activation(self.rotation)

    def get_scale(self):
        return self.scale_activation(self.scale)

    def get_density(self):
        return self.density_activation(self.density)

    def get_features(self):
        return self.features

    def get_shading_normal(self):
        return F.normalize(self.shading_normal, dim=-1)

    def get_material_albedo(self):
        return torch.sigmoid(self.albedo)

    def get_material_roughness(self):
        return torch.sigmoid(self.roughness)

    def get_material_metallic(self):
        return torch.sigmoid(self.metallic)

    def get_environment(self):
        return None if self.environment is None else torch.exp(self.environment)

    def background(self, t2w, dirs, rgb, opacity, train):
        return rgb + (1.0 - opacity) * (self.bg * (1.5 if train else 1.0) + 0.1 * dirs), opacity


class Batch:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def make_batch(h=6, w=5, seed=1, intrinsics="vector", pixel_coords=True, mask=False, lights=False):
    g = torch.Generator().manual_seed(seed)
    fx, fy, cx, cy = 7.0, 6.5, w / 2.0, h / 2.0
    ys, xs = torch.meshgrid(torch.arange(h, dtype=torch.float32), torch.arange(w, dtype=torch.float32), indexing="ij")
    px = torch.stack([xs + 0.5, ys + 0.5], -1).unsqueeze(0)
    d = torch.stack([(px[..., 0] - cx) / fx, (px[..., 1] - cy) / fy, torch.ones(1, h, w)], -1)
    kw = dict(rays_ori=(torch.randn(1, 1, 1, 3, generator=g) * 0.1).expand(1, h, w, 3).clone(),
              rays_dir=F.normalize(d, dim=-1), T_to_world=torch.eye(4).unsqueeze(0) + 0.01 * torch.randn(1, 4, 4,
                                                                                                          generator=g))
    if pixel_coords:
        kw["pixel_coords"] = px
    if intrinsics == "vector":
        kw["intrinsics"] = [fx, fy, cx, cy]
    elif intrinsics == "matrix":
        kw["intrinsics"] = torch.tensor([[fx, 0.0, cx], [0.0, fy, cy], [0.0, 0.0, 1.0]])
    elif intrinsics == "opencv":
        kw["intrinsics_OpenCVPinholeCameraModelParameters"] = dict(
            focal_length=[fx, fy], principal_point=[cx, cy], radial_coeffs=[0.0] * 6, tangential_coeffs=[0.0, 0.0])
    elif intrinsics == "distorted":
        kw["intrinsics_OpenCVPinholeCameraModelParameters"] = dict(
            focal_length=[fx, fy], principal_point=[cx, cy], radial_coeffs=[0.05, 0.0])
    if mask:
        kw["mask"] = (torch.rand(1, h, w, 1, generator=g) > 0.3).float()
    if lights:
        kw["lights"] = torch.rand(2, 9, generator=g)
        kw["light_alias_table"] = torch.rand(5, 3, generator=g)
        kw["mesh_light_vertices"] = torch.rand(3, 3, generator=g)
        kw["mesh_light_triangles"] = torch.tensor([[0, 1, 2]], dtype=torch.int64)
        kw["mesh_lights"] = torch.rand(1, 8, generator=g)
        kw["mesh_light_triangle_alias_table"] = torch.rand(3, 1, generator=g)
    return Batch(**kw)


def make_conf(render_spp=1, inversion_spp=1, spp_chunk=None, filter_type="none", hide=False, lambda_light=0.0,
              max_update=4, clamping=False, max_bounces=3):
    r = AttrDict(pipeline_type="reference", backward_pipeline_type="referenceBwd", primitive_type="instances",
                 particle_kernel_degree=2, particle_kernel_min_response=0.0113,
                 particle_kernel_density_clamping=clamping, particle_radiance_sph_degree=1, enable_normals=True,
                 enable_hitcounts=True, enable_mis=True, enable_kernel_timings=False, render_spp=render_spp,
                 inversion_spp=inversion_spp, filter_type=filter_type, hide_intermediate_outputs=hide,
                 min_transmittance=0.001, max_bounces=max_bounces, max_consecutive_bvh_update=max_update)
    if spp_chunk is not None:
        r["spp_chunk"] = spp_chunk
    return AttrDict(render=r, model=AttrDict(optimize_material_metallic=True),
                    loss=AttrDict(lambda_light=lambda_light))


# (name, conf kwargs, batch kwargs, model kwargs, render kwargs)
CASES = [
    ("spp1_eval", dict(render_spp=1), dict(), dict(), dict(train=False, frame_id=0)),
    ("spp4_chunk2_train_hidden", dict(inversion_spp=4, spp_chunk=2, hide=True, lambda_light=0.5), dict(lights=True),
     dict(), dict(train=True, frame_id=3)),
    ("spp3_chunk2_opencv_atrous_mask", dict(render_spp=3, spp_chunk=2, filter_type="atrous"),
     dict(intrinsics="opencv", mask=True), dict(), dict(train=False, frame_id=7, sh_indirect=True)),
    ("spp8_matrix_no_env", dict(inversion_spp=8), dict(intrinsics="matrix"), dict(environment=False, alias=False),
     dict(train=True, frame_id=11)),
    ("spp5_chunk3_train", dict(inversion_spp=5, spp_chunk=3, max_bounces=2), dict(mask=True), dict(alias=False),
     dict(train=True, frame_id=2)),
    ("spp2_no_pixel_coords", dict(render_spp=2), dict(pixel_coords=False), dict(), dict(train=False, frame_id=1)),
    ("spp2_distorted", dict(render_spp=2), dict(intrinsics="distorted"), dict(), dict(train=False, frame_id=1)),
]

# build_acc sequence: (rebuild flag) per call, under max_consecutive_bvh_update = 3
BUILD_SEQUENCE = [True, False, False, False, False, True, False]


@contextmanager
def cpu_context():
    """Both tracers create a CUDA context with torch.zeros(1, device="cuda") in their constructor;
    on a machine without a GPU that tensor is made on the CPU instead."""
    orig = torch.zeros

    def zeros(*a, **k):
        if k.get("device") == "cuda" and not torch.cuda.is_available():
            k["device"] = "cpu"
        return orig(*a, **k)

    torch.zeros = zeros
    try:
        yield
    finally:
        torch.zeros = orig


def run_case(tracer_cls, case):
    """Renders `case` with `tracer_cls` (whose plugin is a RecordingPlugin) and back-propagates a
    seeded weighted sum of every image output. Returns a flat {name: tensor} record."""
    name, ck, bk, mk, rk = case
    torch.manual_seed(1234)
    with cpu_context():
        tr = tracer_cls(make_conf(**ck))
    plugin = tr.tracer_wrapper
    model = Gaussians(**mk)
    batch = make_batch(**bk)
    out = tr.render(model, batch, **rk)
    rec = {}
    g = torch.Generator().manual_seed(99)
    loss = torch.zeros(())
    for k in sorted(out):
        v = out[k]
        if not isinstance(v, torch.Tensor):
            rec[f"out/{k}"] = torch.tensor([float(v)])
            continue
        rec[f"out/{k}"] = v.detach().clone()
        if v.requires_grad:
            loss = loss + (v * torch.randn(v.shape, generator=g)).sum()
    loss.backward()
    pnames = ["positions", "rotation", "scale", "density", "features", "shading_normal", "albedo", "roughness",
              "metallic", "environment"]
    for pn, p in zip(pnames, model.params()):
        rec[f"grad/{pn}"] = p.grad.clone() if p.grad is not None else torch.zeros(0)
    for i, (method, tensors, scalars) in enumerate(plugin.calls):
        rec[f"call{i}/{method}/scalars"] = torch.tensor(scalars, dtype=torch.float64)
        for j, t in enumerate(tensors):
            rec[f"call{i}/{method}/t{j}"] = t
    return rec


def run_build_sequence(tracer_cls):
    with cpu_context():
        tr = tracer_cls(make_conf(max_update=3))
    model = Gaussians()
    for rebuild in BUILD_SEQUENCE:
        tr.build_acc(model, rebuild=rebuild)
    rec = {}
    for i, (method, tensors, scalars) in enumerate(tr.tracer_wrapper.calls):
        rec[f"call{i}/{method}/scalars"] = torch.tensor(scalars, dtype=torch.float64)
        for j, t in enumerate(tensors):
            rec[f"call{i}/{method}/t{j}"] = t.detach()
    return rec


def constructor_args(tracer_cls):
    with cpu_context():
        tr = tracer_cls(make_conf())
    return [float(a) if isinstance(a, (bool, int, float)) else str(a) for a in tr.tracer_wrapper.ctor[2:]]


__all__ = ["AttrDict", "RecordingPlugin", "Gaussians", "make_batch", "make_conf", "CASES", "run_case",
           "run_build_sequence", "constructor_args", "cpu_context"]
