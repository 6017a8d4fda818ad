"""Point, sphere and triangle-mesh lights: the CUDA tracer (through the C ABI) against the FP64
oracle on seeded scenes.

The light tables come from ptir_b200.lights (pinned to the reference's own table builders by
tests/test_lights.py). Cases cover the top-level light table with and without the environment
in it, lights seen directly by escaped rays (render.visualize_lights), both schedules, the
INDIRECT render mode and the adjoint. Tolerances are those of the environment-only parity tests:
per-sample outputs within 1e-3 + 1e-3 |oracle| on >= 99 % of samples, image means within 1 %, and
gradients as whole vectors within relative L2 2e-3 / cosine 0.999. With exact_replay the albedo
gradient under a point light matches FP64 central differences of the oracle's forward; the
reference's adjoint, which weights the light-sample term by the (here absent) environment, does
not.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from ptir_b200 import synthetic
from tests.golden.make_golden import light_case
from tests.scenes import gpu_trace, gpu_trace_bwd, make_tracer, small_scene, to_torch, with_lights

pytestmark = pytest.mark.gpu


def _close_frac(a, b, atol=1e-3, rtol=1e-3):
    a = a.reshape(-1, a.shape[-1] if a.ndim > 3 else 1)
    b = b.reshape(a.shape)
    return float(np.all(np.abs(a - b) <= atol + rtol * np.abs(b), axis=1).mean())


def _rel_cos(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
    cos = float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))
    return rel, cos


def _outputs(res):
    names = ("radiance", "density", "hit", "hit2", "distortion", "normal", "snormal", "material", "hits_count",
             "visibility", "pbr", "light", "components")
    return {k: v.detach().cpu().numpy() for k, v in zip(names, res)}


def _scene(case):
    lights, _, _ = light_case(case["lights"])
    s = small_scene(n=case.get("n", 2000), w=40, h=32, spp=2, max_bounces=case.get("bounces", 3),
                    env=case.get("env", True), seed=case.get("seed", 0))
    s = with_lights(s, lights, environment=case.get("env", True))
    s["render_opts"] = case.get("render_opts", 0)
    return s


CASES = [
    dict(lights="mixed", env=True),
    dict(lights="mixed", env=False, visualize=True),
    dict(lights="mixed", env=True, visualize=True, render_opts=1),
    dict(lights="point_only", env=False, bounces=2),
    dict(lights="cube_sphere", env=True, seed=3),
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("schedule", ["wavefront", "megakernel"])
def test_forward_with_lights(cuda_device, case, schedule):
    s = _scene(case)
    visualize = case.get("visualize", False)
    ref, vis_ref, st_ref = O.trace(O.OracleConfig(visualize_lights=visualize), s, "f64")
    assert float(np.abs(ref["pbr"]).sum()) > 0.0
    tr = make_tracer(schedule=schedule, visualize=visualize)
    out = _outputs(gpu_trace(tr, to_torch(s)))
    torch.cuda.synchronize()
    assert tr.device_status() == 0
    for k in ("radiance", "density", "material"):
        assert _close_frac(out[k], ref[k]) >= 0.995, k
    for k in ("pbr", "light", "components"):
        frac = _close_frac(out[k], ref[k])
        assert frac >= 0.99, (k, frac)
        m_ref, m_gpu = float(ref[k].mean()), float(out[k].mean())
        assert abs(m_gpu - m_ref) <= 1e-2 * max(abs(m_ref), 1e-3) + 1e-4, (k, m_gpu, m_ref)
    c = tr.counters()
    assert abs(c["segments"] - st_ref.segments) <= 0.01 * st_ref.segments


def test_lights_change_the_image(cuda_device):
    """The same scene without its lights renders differently (the tables are read)."""
    s = _scene(dict(lights="mixed", env=True))
    tr = make_tracer()
    with_l = _outputs(gpu_trace(tr, to_torch(s)))["pbr"]
    bare = {k: v for k, v in s.items() if not k.startswith(("lights", "light_", "mesh_"))}
    without = _outputs(gpu_trace(tr, to_torch(bare)))["pbr"]
    assert float(np.abs(with_l - without).mean()) > 1e-3 * float(np.abs(without).mean())


@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[3]])
@pytest.mark.parametrize("schedule", ["wavefront", "megakernel"])
def test_backward_with_lights(cuda_device, case, schedule):
    s = _scene(case)
    visualize = case.get("visualize", False)
    cfg = O.OracleConfig(visualize_lights=visualize)
    ref, _, _ = O.trace(cfg, s, "f64")
    rng = np.random.default_rng(5)
    zhw = s["ray_ori"].shape[:3]
    grads = dict(pbr=rng.standard_normal(zhw + (3,)).astype(np.float32),
                 light=0.1 * rng.standard_normal(zhw + (3,)).astype(np.float32),
                 material=rng.standard_normal(zhw + (5,)).astype(np.float32))
    mg_ref, eg_ref, _ = O.trace_bwd(cfg, s, ref, grads, "f64")
    tr = make_tracer(schedule=schedule, visualize=visualize)
    S = to_torch(s)
    fwd = list(gpu_trace(tr, S))
    fwd[10] = torch.from_numpy(ref["pbr"]).cuda()
    fwd[11] = torch.from_numpy(ref["light"]).cuda()
    g = {k: torch.from_numpy(v).cuda() for k, v in grads.items()}
    _, mg, _, _, eg = gpu_trace_bwd(tr, S, fwd, g["pbr"], g["light"], g["material"])
    torch.cuda.synchronize()
    assert tr.device_status() == 0
    rel, cos = _rel_cos(mg.cpu().numpy()[:, :4], mg_ref[:, :4])
    assert rel <= 2e-3 and cos >= 0.999, ("material", rel, cos)
    if case.get("env", True):
        rel, cos = _rel_cos(eg.cpu().numpy()[..., :3], eg_ref[..., :3])
        assert rel <= 2e-3 and cos >= 0.999, ("environment", rel, cos)


def test_point_light_albedo_gradient_matches_central_differences(cuda_device):
    # the light sits between the camera and the field, so that surfaces the camera sees are lit
    eye = synthetic.camera_positions(1, seed=0)[0]
    light = dict(type="point", position=tuple(0.7 * eye + np.array([0.3, 0.2, 0.1])), intensity=(6.0, 5.0, 4.0))
    s = with_lights(small_scene(n=1500, w=32, h=24, spp=2, max_bounces=2, scale_range=(0.03, 0.12), env=False),
                    [light], environment=False)
    rng = np.random.default_rng(8)
    W = rng.standard_normal(s["ray_ori"].shape[:3] + (3,)).astype(np.float32)
    ref, vis, _ = O.trace(O.OracleConfig(), s, "f64")
    assert float(np.abs(ref["pbr"]).sum()) > 0.0
    visible = np.nonzero(vis != 0)[0]
    ids = rng.choice(visible, size=min(48, visible.size), replace=False)
    params = [(int(i), int(rng.integers(0, 3))) for i in ids]

    def loss(scene):
        out, _, _ = O.trace(O.OracleConfig(), scene, "f64")
        return float(np.sum(out["pbr"].astype(np.float64) * W))

    fd = []
    for i, c in params:
        mp, mm = s["material"].copy(), s["material"].copy()
        a = mp[i, c]
        mp[i, c] = np.float32(a + 1e-4)
        mm[i, c] = np.float32(a - 1e-4)
        fd.append((loss(dict(s, material=mp)) - loss(dict(s, material=mm))) / (float(mp[i, c]) - float(mm[i, c])))
    fd = np.array(fd)
    S = to_torch(s)
    grads = {}
    for exact in (True, False):
        tr = make_tracer(exact_replay=exact)
        fwd = list(gpu_trace(tr, S))
        fwd[10] = torch.from_numpy(ref["pbr"]).cuda()
        fwd[11] = torch.from_numpy(ref["light"]).cuda()
        mg = gpu_trace_bwd(tr, S, fwd, torch.from_numpy(W).cuda())[1].cpu().numpy()
        grads[exact] = np.array([mg[i, c] for i, c in params], np.float64)
        assert tr.device_status() == 0
    rel, cos = _rel_cos(grads[True], fd)
    assert cos >= 0.995 and rel <= 3e-2, (rel, cos)
    rel_ref, _ = _rel_cos(grads[False], fd)
    assert rel_ref > 10 * rel, (rel_ref, rel)


def test_light_table_validation(cuda_device):
    s = _scene(dict(lights="mixed", env=True))
    S = to_torch(s)
    tr = make_tracer()
    bad = dict(S, lights=S["lights"][:, :8].contiguous())
    with pytest.raises(ValueError):
        gpu_trace(tr, bad)
    bad = dict(S, mesh_light_triangles=S["mesh_light_triangles"].float())
    with pytest.raises(TypeError):
        gpu_trace(tr, bad)
