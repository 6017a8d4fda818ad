"""The adjoint against FP64 central differences of the forward.

The loss is L = sum(pbr * W) for a fixed random W. Path decisions (acceptance, shadow and
transmission draws, BRDF lobes and directions) do not depend on albedo or on environment texels,
so with the sample sequence held fixed L is a smooth function of them, and the FP64 oracle's
central differences (h = 1e-4, divided by the perturbation actually stored in float32) give its
derivative. The GPU adjoint with exact_replay (the re-traversals include each segment's last
composited Gaussian, which the reference's float epsilon leaves out) must match them on 64
random albedo parameters: cosine >= 0.995 and relative L2 <= 3e-2 (the FP32 kernels branch
differently from FP64 on a few paths). The reference-faithful adjoint (exact_replay off) is at
least as far from the differences.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.scenes import gpu_trace, gpu_trace_bwd, make_tracer, small_scene, to_torch

pytestmark = pytest.mark.gpu


def _loss(scene, W):
    out, _, _ = O.trace(O.OracleConfig(), scene, "f64")
    return float(np.sum(out["pbr"].astype(np.float64) * W))


def _fd(scene, W, params, h=1e-4):
    """Central differences of the loss in each (gaussian, channel) albedo parameter."""
    g = np.zeros(len(params))
    for k, (i, c) in enumerate(params):
        mat = scene["material"]
        a = mat[i, c]
        plus, minus = dict(scene), dict(scene)
        mp, mm = mat.copy(), mat.copy()
        mp[i, c] = np.float32(a + h)
        mm[i, c] = np.float32(a - h)
        plus["material"], minus["material"] = mp, mm
        g[k] = (_loss(plus, W) - _loss(minus, W)) / (float(mp[i, c]) - float(mm[i, c]))
    return g


def test_albedo_gradient_matches_central_differences(cuda_device):
    s = small_scene(n=1500, w=32, h=24, spp=2, max_bounces=3, scale_range=(0.03, 0.12))
    rng = np.random.default_rng(21)
    zhw = s["ray_ori"].shape[:3]
    W = rng.standard_normal(zhw + (3,)).astype(np.float32)
    ref, vis, _ = O.trace(O.OracleConfig(), s, "f64")
    # parameters of Gaussians that contribute to the image
    visible = np.nonzero(vis != 0)[0]
    ids = rng.choice(visible, size=min(64, visible.size), replace=False)
    params = [(int(i), int(rng.integers(0, 3))) for i in ids]
    fd = _fd(s, W.astype(np.float64), params)

    S = to_torch(s)
    grads = {}
    for exact in (True, False):
        tr = make_tracer(exact_replay=exact)
        fwd = list(gpu_trace(tr, S))
        fwd[10] = torch.from_numpy(ref["pbr"]).cuda()
        fwd[11] = torch.from_numpy(ref["light"]).cuda()
        mg = gpu_trace_bwd(tr, S, fwd, torch.from_numpy(W).cuda())[1].cpu().numpy()
        grads[exact] = np.array([mg[i, c] for i, c in params], np.float64)
        torch.cuda.synchronize()
        assert tr.device_status() == 0

    def rel_cos(a, b):
        return np.linalg.norm(a - b) / np.linalg.norm(b), float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))

    rel, cos = rel_cos(grads[True], fd)
    assert cos >= 0.995 and rel <= 3e-2, (rel, cos)
    rel_ref, _ = rel_cos(grads[False], fd)
    assert rel_ref >= rel - 1e-6, (rel_ref, rel)
