"""16-bit attribute storage (BF16 / FP16): parity with the FP64 oracle on the rounded attributes.

A tracer with 16-bit storage rounds the Gaussians' geometry, material, shading normals and SH to
the storage type (nearest even) and computes in FP32. Fed the same rounded attributes, the FP64
oracle must agree with it to the tolerances of the FP32 path: per-sample primary outputs within
1e-3 + 1e-3|oracle| on >= 99.5 % of samples, PBR / light on >= 99 %, gradients rel-L2 <= 2e-3 and
cosine >= 0.999. The error of the rounding itself (against the oracle on the unrounded
attributes) is reported by the storage benchmark, not bounded here beyond a sanity check.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.scenes import gpu_trace, gpu_trace_bwd, make_tracer, round_scene, small_scene, to_torch

pytestmark = pytest.mark.gpu

NAMES = ("radiance", "density", "hit", "hit2", "distortion", "normal", "snormal", "material", "hits_count",
         "visibility", "pbr", "light", "components")


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


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
@pytest.mark.parametrize("schedule", ["wavefront", "megakernel"])
def test_forward_matches_oracle_on_rounded_attributes(cuda_device, storage, schedule):
    s = small_scene(n=3000, w=40, h=32, spp=2, max_bounces=3, sh_full=True)
    ref, vis_ref, _ = O.trace(O.OracleConfig(), round_scene(s, storage), "f64")
    tr = make_tracer(schedule=schedule, storage=storage)
    out = {k: v.detach().cpu().numpy() for k, v in zip(NAMES, gpu_trace(tr, to_torch(s)))}
    torch.cuda.synchronize()
    assert tr.device_status() == 0
    for k in ("radiance", "density", "hit", "hit2", "distortion", "normal", "snormal", "material", "hits_count"):
        assert _close_frac(out[k], ref[k]) >= 0.995, (k, storage)
    for k in ("pbr", "light", "components"):
        assert _close_frac(out[k], ref[k]) >= 0.99, (k, storage)
    vg = out["visibility"].reshape(-1).view(np.int32) != 0
    assert (vg != (vis_ref != 0)).sum() <= max(2, 0.005 * (vis_ref != 0).sum())
    # sanity: the rounding moves the image by little against the unrounded scene
    full, _, _ = O.trace(O.OracleConfig(), s, "f64")
    assert np.abs(out["radiance"] - full["radiance"]).mean() < 2e-2


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
def test_backward_matches_oracle_on_rounded_attributes(cuda_device, storage):
    s = small_scene(n=2000, w=40, h=32, spp=2, max_bounces=3)
    r = round_scene(s, storage)
    cfg = O.OracleConfig()
    ref, _, _ = O.trace(cfg, r, "f64")
    rng = np.random.default_rng(5)
    zhw = s["ray_ori"].shape[:3]
    grads = dict(pbr=rng.standard_normal(zhw + (3,)).astype(np.float32),
                 light=0.1 * rng.standard_normal(zhw + (3,)).astype(np.float32),
                 material=rng.standard_normal(zhw + (5,)).astype(np.float32))
    mg_ref, eg_ref, _ = O.trace_bwd(cfg, r, ref, grads, "f64")
    tr = make_tracer(storage=storage)
    S = to_torch(s)
    fwd = list(gpu_trace(tr, S))
    fwd[10] = torch.from_numpy(ref["pbr"]).cuda()
    fwd[11] = torch.from_numpy(ref["light"]).cuda()
    g = {k: torch.from_numpy(v).cuda() for k, v in grads.items()}
    _, mg, _, _, eg = gpu_trace_bwd(tr, S, fwd, g["pbr"], g["light"], g["material"])
    torch.cuda.synchronize()
    assert tr.device_status() == 0
    rel, cos = _rel_cos(mg.cpu().numpy()[:, :4], mg_ref[:, :4])
    assert rel <= 2e-3 and cos >= 0.999, ("material", storage, rel, cos)
    rel, cos = _rel_cos(eg.cpu().numpy()[..., :3], eg_ref[..., :3])
    assert rel <= 2e-3 and cos >= 0.999, ("environment", storage, rel, cos)


def test_fp32_storage_reads_caller_tensors(cuda_device):
    """FP32 storage and BF16 storage of attributes that are already BF16 values give the same image."""
    s = round_scene(small_scene(n=1500, w=32, h=24, spp=1), "bf16")
    S = to_torch(s)
    a = [t.clone() for t in gpu_trace(make_tracer(storage="fp32"), S)]
    b = gpu_trace(make_tracer(storage="bf16"), S)
    for k, (x, y) in enumerate(zip(a, b)):
        if k == 9:
            assert torch.equal(x.view(torch.int32), y.view(torch.int32))
        else:
            assert torch.isclose(x, y, rtol=1e-5, atol=1e-6).float().mean().item() >= 0.999, NAMES[k]


def test_ray_order_does_not_change_results(cuda_device):
    """Sorting bounce rays only reorders independent segments: outputs agree with queue order
    (visibility flags exactly, the rest up to float32 atomic order in the backward)."""
    s = small_scene(n=2500, w=40, h=36, spp=2, max_bounces=4)
    S = to_torch(s)
    outs = []
    for sort in (True, False):
        outs.append([t.clone() for t in gpu_trace(make_tracer(sort_rays=sort), S)])
    for k, (x, y) in enumerate(zip(*outs)):
        if k == 9:
            assert torch.equal(x.view(torch.int32), y.view(torch.int32))
        else:
            assert torch.equal(x, y), NAMES[k]
