"""``SelectiveAdam``: the reference's fused selective Adam (threedgrut/optimizers/__init__.py:45-125)
on the library's sm_100a kernel (``ptir_selective_adam``).

Same constructor (params, lr, betas, eps), same ``step(visibility)`` and the same update: for the
rows (Gaussians) whose visibility is set, ``m = b1 m + (1-b1) g``, ``v = b2 v + (1-b2) g^2``,
``p -= lr m / (sqrt(v) + eps)``, without bias correction; hidden rows keep parameter and moments.
"""
from __future__ import annotations

import torch

from . import _native as N


class SelectiveAdam(torch.optim.Adam):
    def __init__(self, params, lr=0.001, betas=(0.9, 0.999), eps=1e-08):
        super().__init__(params=params, lr=lr, eps=eps, betas=betas)
        self._lib = N.load()

    @torch.no_grad()
    def step(self, visibility):
        for group in self.param_groups:
            lr, eps = group["lr"], group["eps"]
            beta1, beta2 = group["betas"]
            if len(group["params"]) != 1:
                raise ValueError("More than one tensor in group is not supported")
            param = group["params"][0]
            if param.grad is None:
                continue
            state = self.state[param]
            if len(state) == 0:
                state["step"] = torch.tensor(0.0, dtype=torch.float32)
                state["exp_avg"] = torch.zeros_like(param, memory_format=torch.preserve_format)
                state["exp_avg_sq"] = torch.zeros_like(param, memory_format=torch.preserve_format)
            state["step"] += 1
            if param.dtype != torch.float32 or not param.is_cuda or not param.is_contiguous():
                raise TypeError("SelectiveAdam: contiguous float32 CUDA parameters required")
            grad = param.grad.contiguous()
            n = param.shape[0] if param.dim() > 0 else 1
            row = param.numel() // max(n, 1)
            vis = None
            if visibility is not None:
                vis = (visibility.reshape(-1)[:n] != 0).to(device=param.device, dtype=torch.uint8).contiguous()
            rc = self._lib.ptir_selective_adam(
                param.data_ptr(), grad.data_ptr(), state["exp_avg"].data_ptr(), state["exp_avg_sq"].data_ptr(),
                None if vis is None else vis.data_ptr(), int(n), int(max(row, 1)), float(lr), float(beta1),
                float(beta2), float(eps), torch.cuda.current_stream(param.device).cuda_stream)
            if rc != N.PTIR_OK:
                raise N.PtirError(rc, "ptir_selective_adam failed")


def selective_adam_(param: torch.Tensor, grad: torch.Tensor, exp_avg: torch.Tensor, exp_avg_sq: torch.Tensor,
                    visible: torch.Tensor | None, lr: float, beta1: float = 0.9, beta2: float = 0.999,
                    eps: float = 1e-8) -> None:
    """In-place fused step on raw [N, ...] float32 CUDA tensors (visible: [N] uint8 / bool, or None)."""
    n = param.shape[0]
    row = param.numel() // max(n, 1)
    vis = None if visible is None else visible.to(torch.uint8).contiguous()
    rc = N.load().ptir_selective_adam(param.data_ptr(), grad.data_ptr(), exp_avg.data_ptr(), exp_avg_sq.data_ptr(),
                                      None if vis is None else vis.data_ptr(), int(n), int(max(row, 1)), float(lr),
                                      float(beta1), float(beta2), float(eps),
                                      torch.cuda.current_stream(param.device).cuda_stream)
    if rc != N.PTIR_OK:
        raise N.PtirError(rc, "ptir_selective_adam failed")
