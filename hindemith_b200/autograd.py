"""Differentiable Horn-Schunck: ``horn_schunck(I0, I1, alpha, iters)`` -> (u, v) whose
backward gives dL/dI0, dL/dI1 and dL/dalpha through the hand-written adjoint kernels
(libhsflow's hs_forward_train / hs_backward).  The forward keeps (u, v) every
`ckpt_every` sweeps; the backward recomputes each interval from its checkpoint and
runs the adjoint sweeps in reverse.  `alpha` may be a CUDA tensor (learnable; it stays
on the device) or a number.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib as L
from . import device as D


def _plane_like(t: torch.Tensor, ld: int) -> torch.Tensor:
    """`t` (H, W) as a float32 plane with row stride ld."""
    H, W = t.shape
    if D.is_plane(t) and t.stride(0) == ld:
        return t
    p = torch.empty((H, ld), dtype=torch.float32, device=t.device)[:, :W]
    p.copy_(t)
    return p


class HornSchunckFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, I0, I1, alpha, iters: int, ckpt_every: int, config: Optional[L.hs_config]):
        cfg = config if config is not None else L.make_config()
        I0p, I1p = D._same_layout(I0.detach(), I1.detach())
        H, W = I0p.shape
        ld = I0p.stride(0)
        dev = I0p.device
        a = alpha.detach().to(device=dev, dtype=torch.float32).reshape(1).contiguous()
        lib = L.lib()
        uv = torch.empty((2, H, ld), dtype=torch.float32, device=dev)[:, :, :W]
        derivs = torch.empty(lib.hs_derivs_bytes(H, W, ld), dtype=torch.uint8, device=dev)
        ckpt = torch.empty(max(lib.hs_checkpoint_bytes(H, W, ld, iters, ckpt_every), 256),
                           dtype=torch.uint8, device=dev)
        ws = D.workspace(lib.hs_forward_train_workspace_bytes(H, W, ld), dev)
        L.check(lib.hs_forward_train(D.ptr(I0p), D.ptr(I1p), H, W, ld, D.ptr(a), int(iters),
                                     int(ckpt_every), D.ptr(uv[0]), D.ptr(uv[1]), D.ptr(derivs),
                                     D.ptr(ckpt), D.ptr(ws), ws.numel(), ctypes.byref(cfg),
                                     D.stream_handle()), "hs_forward_train")
        ctx.save_for_backward(derivs, ckpt, a)
        ctx.meta = (H, W, ld, int(iters), int(ckpt_every), cfg, alpha.shape, alpha.dtype)
        return uv[0], uv[1]

    @staticmethod
    def backward(ctx, gu, gv):
        derivs, ckpt, a = ctx.saved_tensors
        H, W, ld, iters, ckpt_every, cfg, ashape, adtype = ctx.meta
        dev = derivs.device
        if gu is None:
            gu = torch.zeros((H, W), device=dev)
        if gv is None:
            gv = torch.zeros((H, W), device=dev)
        gu = _plane_like(gu.to(torch.float32), ld)
        gv = _plane_like(gv.to(torch.float32), ld)
        lib = L.lib()
        out = torch.empty((2, H, ld), dtype=torch.float32, device=dev)[:, :, :W]
        dalpha = torch.zeros(1, dtype=torch.float32, device=dev)
        ws = torch.empty(lib.hs_backward_workspace_bytes(H, W, ld, ckpt_every), dtype=torch.uint8,
                         device=dev)
        L.check(lib.hs_backward(D.ptr(derivs), H, W, ld, D.ptr(a), iters, ckpt_every, D.ptr(ckpt),
                                D.ptr(gu), D.ptr(gv), D.ptr(out[0]), D.ptr(out[1]),
                                D.ptr(dalpha), D.ptr(ws), ws.numel(), ctypes.byref(cfg),
                                D.stream_handle()), "hs_backward")
        da = dalpha.reshape(ashape).to(adtype) if ctx.needs_input_grad[2] else None
        return out[0], out[1], da, None, None, None


def horn_schunck(I0: torch.Tensor, I1: torch.Tensor, alpha, iters: int, ckpt_every: int = 10,
                 config: Optional[L.hs_config] = None):
    """Differentiable plain Horn-Schunck forward -> (u, v)."""
    if not isinstance(alpha, torch.Tensor):
        alpha = torch.tensor(float(alpha), dtype=torch.float32, device=I0.device)
    return HornSchunckFunction.apply(I0, I1, alpha, int(iters), int(ckpt_every), config)
