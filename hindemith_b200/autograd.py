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


class HornSchunckBatchFunction(torch.autograd.Function):
    """n pairs (each its own size) sharing one alpha; one launch per pass for all pairs."""

    @staticmethod
    def forward(ctx, alpha, iters: int, ckpt_every: int, config, *images):
        cfg = config if config is not None else L.make_config()
        n = len(images) // 2
        if n < 1 or n > L.HS_MAX_TRAIN_PAIRS:
            raise ValueError(f"1..{L.HS_MAX_TRAIN_PAIRS} pairs per batch, got {n}")
        dev = images[0].device
        a = alpha.detach().to(device=dev, dtype=torch.float32).reshape(1).contiguous()
        descs = (L.hs_train_pair * n)()
        keep, outs = [], []
        for i in range(n):
            I0p, I1p = D._same_layout(images[2 * i].detach(), images[2 * i + 1].detach())
            H, W = I0p.shape
            uv = torch.empty((2, H, I0p.stride(0)), dtype=torch.float32, device=dev)[:, :, :W]
            d = descs[i]
            d.I0, d.I1, d.u, d.v = I0p.data_ptr(), I1p.data_ptr(), uv[0].data_ptr(), uv[1].data_ptr()
            d.alpha = a.data_ptr()
            d.H, d.W, d.ld, d.reserved = H, W, I0p.stride(0), 0
            keep += [I0p, I1p]
            outs += [uv[0], uv[1]]
        lib = L.lib()
        nbytes = lib.hs_train_workspace_bytes(descs, n, int(iters), int(ckpt_every))
        if nbytes == 0:
            raise L.HSError(L.HS_ERR_INVALID_ARG, "hs_train_workspace_bytes", "invalid batch")
        ws = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
        L.check(lib.hs_forward_train_batched(descs, n, int(iters), int(ckpt_every), D.ptr(ws),
                                             ws.numel(), ctypes.byref(cfg), D.stream_handle()),
                "hs_forward_train_batched")
        ctx.state = (descs, ws, a, int(iters), int(ckpt_every), cfg, keep)
        ctx.alpha_shape, ctx.alpha_dtype = alpha.shape, alpha.dtype
        return tuple(outs)

    @staticmethod
    def backward(ctx, *grads):
        descs, ws, a, iters, ckpt_every, cfg, keep = ctx.state
        n = len(grads) // 2
        dev = ws.device
        dalpha = torch.zeros(n, dtype=torch.float32, device=dev)
        gin = []
        for i in range(n):
            d = descs[i]
            H, W, ld = d.H, d.W, d.ld
            gu, gv = grads[2 * i], grads[2 * i + 1]
            gu = torch.zeros((H, W), device=dev) if gu is None else gu
            gv = torch.zeros((H, W), device=dev) if gv is None else gv
            gu, gv = _plane_like(gu.to(torch.float32), ld), _plane_like(gv.to(torch.float32), ld)
            out = torch.empty((2, H, ld), dtype=torch.float32, device=dev)[:, :, :W]
            d.dLdu, d.dLdv = gu.data_ptr(), gv.data_ptr()
            d.dI0, d.dI1 = out[0].data_ptr(), out[1].data_ptr()
            d.dalpha = dalpha.data_ptr() + 4 * i
            gin += [out[0], out[1], gu, gv]
        lib = L.lib()
        L.check(lib.hs_backward_batched(descs, n, iters, ckpt_every, D.ptr(ws), ws.numel(),
                                        ctypes.byref(cfg), D.stream_handle()), "hs_backward_batched")
        da = dalpha.sum().reshape(ctx.alpha_shape).to(ctx.alpha_dtype) if ctx.needs_input_grad[0] else None
        img_grads = []
        for i in range(n):
            img_grads += [gin[4 * i], gin[4 * i + 1]]
        return (da, None, None, None, *img_grads)


def horn_schunck_batch(pairs, alpha, iters: int, ckpt_every: int = 10,
                       config: Optional[L.hs_config] = None):
    """Differentiable Horn-Schunck for a list of (I0, I1) pairs sharing alpha -> [(u, v)]."""
    dev = pairs[0][0].device
    if not isinstance(alpha, torch.Tensor):
        alpha = torch.tensor(float(alpha), dtype=torch.float32, device=dev)
    flat = [t for pr in pairs for t in pr]
    outs = HornSchunckBatchFunction.apply(alpha, int(iters), int(ckpt_every), config, *flat)
    return [(outs[2 * i], outs[2 * i + 1]) for i in range(len(pairs))]
