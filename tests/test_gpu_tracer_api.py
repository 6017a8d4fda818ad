"""The reference-facing Python Tracer (ptir_b200.tracer.Tracer, the drop-in for
threedgptir_tracer/tracer.py's Tracer): render, build_acc, the autograd function and LightBuffers
taken from the batch, on a small seeded scene, against direct OptixTracer calls of the same rays.

The model object is a stand-in with the accessors Tracer reads from threedgrut's model
(positions, get_rotation, get_material_albedo, get_environment, background, ...). With 1 spp
and no filter, render's outputs are the trace outputs plus the reference's post-processing:
pred_pbr, pred_direct and pred_indirect times the opacity, pred_dist divided by it, normals
normalised. The albedo gradient of a loss on pred_pbr is the trace_bwd material gradient for
the pbr gradient the autograd chain hands it (the loss weight times the opacity).
"""
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from ptir_b200 import envmap
from ptir_b200.tracer import Tracer
from tests.golden.make_golden import light_case
from tests.scenes import gpu_trace, gpu_trace_bwd, make_tracer, small_scene, to_torch, with_lights

pytestmark = pytest.mark.gpu


class Model:
    """The part of threedgrut's model surface that Tracer uses."""

    def __init__(self, s, S):
        self.positions = S["build_pos"]
        self.rotation = S["build_rot"]
        self.scale = S["build_scl"]
        self.density = S["build_dns"]
        self.features = S["sph"]
        self.snrm = S["shading_normal"]
        mat = S["material"]
        self.albedo = mat[:, 0:3].clone().requires_grad_(True)
        self.roughness = mat[:, 3:4].clone().requires_grad_(True)
        self.metallic = mat[:, 4:5].clone().requires_grad_(True)
        self.env = S["environment"]
        table = envmap.build(torch.from_numpy(s["environment"]))
        self.environment_alias_table = SimpleNamespace(prob=table["prob"], alias=table["alias"], pdf=table["pdf"],
                                                       height=table["height"], width=table["width"])
        self.n_active_features = 3

    rotation_activation = staticmethod(lambda x: x)
    scale_activation = staticmethod(lambda x: x)
    density_activation = staticmethod(lambda x: x)

    def get_rotation(self):
        return self.rotation

    def get_scale(self):
        return self.scale

    def get_density(self):
        return self.density

    def get_features(self):
        return self.features

    def get_shading_normal(self):
        return self.snrm

    def get_material_albedo(self):
        return self.albedo

    def get_material_roughness(self):
        return self.roughness

    def get_material_metallic(self):
        return self.metallic

    def get_environment(self):
        return self.env

    def background(self, t2w, rays_dir, rgb, opacity, train):
        return rgb, opacity


def _conf(max_bounces):
    r = SimpleNamespace(pipeline_type="reference", backward_pipeline_type="referenceBwd", primitive_type="instances",
                        particle_kernel_degree=4, particle_kernel_min_response=0.0113,
                        particle_kernel_density_clamping=True, particle_radiance_sph_degree=3, enable_normals=True,
                        enable_hitcounts=True, enable_mis=True, min_transmittance=0.001, max_bounces=max_bounces,
                        max_consecutive_bvh_update=1, inversion_spp=1, render_spp=1, filter_type="none",
                        visualize_lights=False)
    return SimpleNamespace(render=r, model=SimpleNamespace(optimize_material_metallic=False), loss=None)


def _scene():
    s = small_scene(n=2000, w=40, h=32, spp=1, max_bounces=3)
    return s, to_torch(s)


def _batch(S, **extra):
    return SimpleNamespace(rays_ori=S["ray_ori"], rays_dir=S["ray_dir"], T_to_world=S["ray_to_world"], **extra)


def test_render_matches_direct_trace(cuda_device):
    s, S = _scene()
    tracer = Tracer(_conf(3))
    model = Model(s, S)
    tracer.build_acc(model, rebuild=True)
    out = tracer.render(model, _batch(S), train=False, frame_id=S["frame"])
    direct = gpu_trace(make_tracer(), S)
    torch.cuda.synchronize()
    rad, dns, hit, _, _, nrm, _, mat, hits, vis, pbr, light, comps = direct
    keys = {"pred_rgb", "pred_opacity", "pred_dist", "pred_depth_second_moment", "pred_depth_distortion",
            "pred_normals", "pred_shadingnormal", "pred_material", "pred_pbr", "pred_light", "pred_direct",
            "pred_indirect", "hits_count", "frame_time_ms", "mog_visibility"}
    assert keys <= set(out), keys - set(out)
    close = lambda a, b: torch.allclose(a, b, rtol=1e-5, atol=1e-6)  # noqa: E731
    assert close(out["pred_rgb"], rad) and close(out["pred_opacity"], dns)
    assert close(out["pred_pbr"], pbr * dns) and close(out["pred_light"], light)
    assert close(out["pred_direct"], comps[..., 0, :] * dns) and close(out["pred_indirect"], comps[..., 1, :] * dns)
    assert close(out["pred_dist"], torch.nan_to_num(hit[..., 0:1] / dns, 0.0, 0.0))
    assert close(out["pred_material"], mat) and close(out["hits_count"], hits)
    assert torch.equal(out["mog_visibility"].view(torch.int32) != 0, vis.view(torch.int32) != 0)
    assert float(pbr.abs().sum()) > 0.0


def test_render_backward_matches_trace_bwd(cuda_device):
    s, S = _scene()
    tracer = Tracer(_conf(3))
    model = Model(s, S)
    tracer.build_acc(model, rebuild=True)
    out = tracer.render(model, _batch(S), train=True, frame_id=S["frame"])
    rng = np.random.default_rng(4)
    W = torch.from_numpy(rng.standard_normal(tuple(out["pred_pbr"].shape)).astype(np.float32)).cuda()
    (out["pred_pbr"] * W).sum().backward()
    torch.cuda.synchronize()
    tr = make_tracer()
    fwd = gpu_trace(tr, S)
    dns = fwd[1]
    _, mg, _, _, _ = gpu_trace_bwd(tr, S, fwd, W * dns)
    torch.cuda.synchronize()
    a = model.albedo.grad.double().reshape(-1)
    b = mg[:, 0:3].double().reshape(-1)
    assert float(b.norm()) > 0.0
    assert float((a - b).norm()) <= 1e-4 * float(b.norm()), float((a - b).norm() / b.norm())
    r = model.roughness.grad.double().reshape(-1)
    assert float((r - mg[:, 3].double()).norm()) <= 1e-4 * float(mg[:, 3].double().norm()) + 1e-12


def test_render_reads_lights_from_the_batch(cuda_device):
    s, S = _scene()
    lights, _, _ = light_case("mixed")
    L = to_torch(with_lights(s, lights, environment=True))
    tracer = Tracer(_conf(3))
    model = Model(s, S)
    tracer.build_acc(model, rebuild=True)
    plain = tracer.render(model, _batch(S), frame_id=S["frame"])["pred_pbr"]
    lit = tracer.render(model, _batch(S, lights=L["lights"], light_alias_table=L["light_alias_table"],
                                      mesh_light_vertices=L["mesh_light_vertices"],
                                      mesh_light_triangles=L["mesh_light_triangles"], mesh_lights=L["mesh_lights"],
                                      mesh_light_triangle_alias_table=L["mesh_light_triangle_alias_table"]),
                        frame_id=S["frame"])["pred_pbr"]
    direct = gpu_trace(make_tracer(), L)
    torch.cuda.synchronize()
    assert torch.allclose(lit.detach(), direct[10] * direct[1], rtol=1e-5, atol=1e-6)
    assert float((lit - plain).detach().abs().mean()) > 0.0
