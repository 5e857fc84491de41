"""Mean end-point error of a batch of flow fields, as one fused libhsflow reduction:

    L = (1/n) sum_i mean_px sqrt((u_i - ut_i)^2 + (v_i - vt_i)^2 + eps)

``mean_epe_batch(flows, targets)`` is differentiable in the flows (the targets are
constants); forward and backward are one launch each for all pairs (plus a one-block fold),
and the sum is deterministic.
"""
from __future__ import annotations

import ctypes
from typing import Sequence, Tuple

import torch

from . import _lib as L
from . import device as D


def _canon(t: torch.Tensor, ld: int) -> torch.Tensor:
    if D.is_plane(t) and t.stride(0) == ld:
        return t
    H, W = t.shape
    p = torch.empty((H, ld), dtype=torch.float32, device=t.device)[:, :W]
    p.copy_(t)
    return p


class MeanEPEBatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eps: float, *planes):
        n = len(planes) // 4
        if n < 1 or n > L.HS_MAX_TRAIN_PAIRS:
            raise ValueError(f"1..{L.HS_MAX_TRAIN_PAIRS} flow fields, got {n}")
        dev = planes[0].device
        descs = (L.hs_epe_pair * n)()
        keep = []
        for i in range(n):
            u, v, ut, vt = (planes[4 * i + q].detach() for q in range(4))
            H, W = u.shape
            if v.shape != (H, W) or ut.shape != (H, W) or vt.shape != (H, W):
                raise ValueError(f"pair {i}: u, v and the targets must have one shape")
            ld = D.padded_ld(W) if not D.is_plane(u) else u.stride(0)
            u, v, ut, vt = (_canon(t.to(torch.float32), ld) for t in (u, v, ut, vt))
            d = descs[i]
            d.u, d.v, d.ut, d.vt = u.data_ptr(), v.data_ptr(), ut.data_ptr(), vt.data_ptr()
            d.du = d.dv = None
            d.H, d.W, d.ld, d.reserved = H, W, ld, 0
            keep += [u, v, ut, vt]
        lib = L.lib()
        ws = torch.empty(int(lib.hs_epe_workspace_bytes(n)), dtype=torch.uint8, device=dev)
        loss = torch.empty((), dtype=torch.float32, device=dev)
        L.check(lib.hs_epe_loss_batched(descs, n, float(eps), D.ptr(loss), D.ptr(ws), ws.numel(),
                                        D.stream_handle()), "hs_epe_loss_batched")
        ctx.state = (descs, keep, float(eps), n)
        return loss

    @staticmethod
    def backward(ctx, gloss):
        descs, keep, eps, n = ctx.state
        g = gloss.detach().to(torch.float32).reshape(()).contiguous()
        grads = []
        for i in range(n):
            d = descs[i]
            buf = torch.empty((2, d.H, d.ld), dtype=torch.float32, device=g.device)[:, :, :d.W]
            d.du, d.dv = buf[0].data_ptr(), buf[1].data_ptr()
            grads += [buf[0], buf[1], None, None]
        L.check(L.lib().hs_epe_loss_backward_batched(descs, n, eps, D.ptr(g), D.stream_handle()),
                "hs_epe_loss_backward_batched")
        return (None, *grads)


def mean_epe_batch(flows: Sequence[Tuple[torch.Tensor, torch.Tensor]],
                   targets: Sequence[Tuple[torch.Tensor, torch.Tensor]],
                   eps: float = 1e-12) -> torch.Tensor:
    """Mean over pairs of the mean end-point error (a 0-d float32 CUDA tensor)."""
    if len(flows) != len(targets):
        raise ValueError("one target per flow field")
    flat = []
    for (u, v), (ut, vt) in zip(flows, targets):
        flat += [u, v, ut, vt]
    return MeanEPEBatch.apply(float(eps), *flat)
