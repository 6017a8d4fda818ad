"""Fused selective Adam against a numpy restatement of the reference's update
(threedgrut/optimizers/optimizers.cu:49-76): two steps with a visibility mask, float32 values
within 1e-6 relative (IEEE square root and division in both)."""
import numpy as np
import pytest
import torch

from ptir_b200.optim import SelectiveAdam

pytestmark = pytest.mark.gpu


def _numpy_steps(p, grads, vis, lr, b1, b2, eps):
    p = p.astype(np.float32).copy()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    f = np.float32
    for g in grads:
        sel = vis[:, None] != 0
        m2 = f(b1) * m + (f(1.0) - f(b1)) * g
        v2 = f(b2) * v + (f(1.0) - f(b2)) * g * g
        step = (-f(lr) * m2) / (np.sqrt(v2) + f(eps))
        p = np.where(sel, p + step, p).astype(np.float32)
        m = np.where(sel, m2, m).astype(np.float32)
        v = np.where(sel, v2, v).astype(np.float32)
    return p, m, v


def test_selective_adam_matches_reference_update(cuda_device):
    rng = np.random.default_rng(3)
    n = 10007
    p0 = rng.standard_normal((n, 5)).astype(np.float32)
    grads = [rng.standard_normal((n, 5)).astype(np.float32) * 1e-2 for _ in range(2)]
    vis = (rng.uniform(size=n) < 0.6).astype(np.uint8)
    param = torch.from_numpy(p0).cuda().requires_grad_(True)
    opt = SelectiveAdam([param], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    for g in grads:
        param.grad = torch.from_numpy(g).cuda()
        opt.step(torch.from_numpy(vis).cuda())
    torch.cuda.synchronize()
    p_ref, m_ref, v_ref = _numpy_steps(p0, grads, vis, 1e-2, 0.9, 0.999, 1e-8)
    st = opt.state[param]
    np.testing.assert_allclose(param.detach().cpu().numpy(), p_ref, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(st["exp_avg"].cpu().numpy(), m_ref, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(st["exp_avg_sq"].cpu().numpy(), v_ref, rtol=1e-6, atol=1e-12)
    hidden = vis == 0
    assert np.array_equal(param.detach().cpu().numpy()[hidden], p0[hidden])
