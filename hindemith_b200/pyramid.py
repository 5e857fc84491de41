"""Coarse-to-fine Horn-Schunck with a reverse mode through the whole pyramid.

Per pair the image pyramid is P_0 = I, P_{l+1} = blur_down(P_l) (5x5 binomial blur,
clamp-to-edge, keep every second pixel).  At the coarsest level the flow is Horn-Schunck
of (P0, P1) from zero; at each finer level the coarser flow is upsampled by 2 (values
doubled), I1 is backward-warped by it with WarpImg2D's rule
(Operations/OpticalFlow/WarpImg2D.cpp:33-75), Horn-Schunck of (P0, warped P1) gives the
increment, and the level's flow is upsampled + increment.  Every step is a libhsflow
kernel (hs_blur_down, hs_upsample2, hs_warp, the batched training sweeps) wrapped in a
torch.autograd.Function whose backward is the matching adjoint kernel, so
``loss.backward()`` runs the adjoint through all levels and the whole forward + backward
can be captured in one CUDA graph (no host synchronisation on the path).
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib as L
from . import device as D
from .autograd import horn_schunck_batch


def _plane(t: torch.Tensor) -> torch.Tensor:
    """`t` as a plane with the canonical padded row stride."""
    H, W = t.shape
    ld = D.padded_ld(W)
    if D.is_plane(t) and t.stride(0) == ld:
        return t
    p = torch.empty((H, ld), dtype=torch.float32, device=t.device)[:, :W]
    p.copy_(t)
    return p


def _new(H: int, W: int, dev) -> torch.Tensor:
    return torch.empty((H, D.padded_ld(W)), dtype=torch.float32, device=dev)[:, :W]


class BlurDown(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        x = _plane(x.detach())
        H, W = x.shape
        out = _new((H + 1) // 2, (W + 1) // 2, x.device)
        L.check(L.lib().hs_blur_down(D.ptr(x), H, W, x.stride(0), D.ptr(out), out.stride(0),
                                     D.stream_handle()), "hs_blur_down")
        ctx.shape = (H, W)
        return out

    @staticmethod
    def backward(ctx, g):
        H, W = ctx.shape
        g = _plane(g.to(torch.float32))
        din = _new(H, W, g.device)
        L.check(L.lib().hs_blur_down_adjoint(D.ptr(g), H, W, din.stride(0), g.stride(0),
                                             D.ptr(din), D.stream_handle()),
                "hs_blur_down_adjoint")
        return din


class Upsample2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, c, H: int, W: int, scale: float):
        c = _plane(c.detach())
        if c.shape != ((H + 1) // 2, (W + 1) // 2):
            raise ValueError(f"coarse shape {tuple(c.shape)} does not halve ({H}, {W})")
        f = _new(H, W, c.device)
        L.check(L.lib().hs_upsample2(D.ptr(c), c.stride(0), D.ptr(f), H, W, f.stride(0),
                                     float(scale), D.stream_handle()), "hs_upsample2")
        ctx.meta = (H, W, float(scale), c.shape)
        return f

    @staticmethod
    def backward(ctx, g):
        H, W, scale, cshape = ctx.meta
        g = _plane(g.to(torch.float32))
        dc = _new(cshape[0], cshape[1], g.device)
        L.check(L.lib().hs_upsample2_adjoint(D.ptr(g), H, W, g.stride(0), D.ptr(dc),
                                             dc.stride(0), scale, D.stream_handle()),
                "hs_upsample2_adjoint")
        return dc, None, None, None


class Warp(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, u, v):
        src, u, v = (_plane(t.detach()) for t in (src, u, v))
        H, W = src.shape
        if u.shape != (H, W) or v.shape != (H, W):
            raise ValueError("src, u and v must have one shape")
        dst = _new(H, W, src.device)
        L.check(L.lib().hs_warp(D.ptr(src), D.ptr(u), D.ptr(v), H, W, src.stride(0), D.ptr(dst),
                                D.stream_handle()), "hs_warp")
        ctx.save_for_backward(src, u, v)
        return dst

    @staticmethod
    def backward(ctx, g):
        src, u, v = ctx.saved_tensors
        H, W = src.shape
        g = _plane(g.to(torch.float32))
        buf = torch.empty((3, H, src.stride(0)), dtype=torch.float32, device=src.device)[:, :, :W]
        lib = L.lib()
        ws = torch.empty(int(lib.hs_warp_adjoint_workspace_bytes(H, W, src.stride(0))),
                         dtype=torch.uint8, device=src.device)
        L.check(lib.hs_warp_adjoint(D.ptr(src), D.ptr(u), D.ptr(v), D.ptr(g), H, W,
                                    src.stride(0), D.ptr(buf[0]), D.ptr(buf[1]),
                                    D.ptr(buf[2]), D.ptr(ws), ws.numel(), D.stream_handle()),
                "hs_warp_adjoint")
        return buf[0], buf[1], buf[2]


def blur_down(x: torch.Tensor) -> torch.Tensor:
    """(ceil(H/2), ceil(W/2)) = every second pixel of the 5x5 binomial blur of x."""
    return BlurDown.apply(x)


def upsample2(c: torch.Tensor, H: int, W: int, scale: float = 2.0) -> torch.Tensor:
    """(H, W) = scale * half-pixel bilinear 2x upsampling of c (ceil(H/2), ceil(W/2))."""
    return Upsample2.apply(c, int(H), int(W), float(scale))


def warp(src: torch.Tensor, u: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """src backward-warped by (u, v) with WarpImg2D's rule."""
    return Warp.apply(src, u, v)


def build_pyramid(img: torch.Tensor, levels: int) -> List[torch.Tensor]:
    pyr = [img]
    for _ in range(levels - 1):
        pyr.append(blur_down(pyr[-1]))
    return pyr


def coarse_to_fine(pairs: Sequence[Tuple[torch.Tensor, torch.Tensor]], alpha, levels: int = 4,
                   iters: int = 100, ckpt_every: int = 10,
                   config: Optional[L.hs_config] = None) -> List[Tuple[torch.Tensor, torch.Tensor]]:
    """Coarse-to-fine Horn-Schunck of each (I0, I1) pair -> [(u, v)] at full resolution.

    `alpha` (a CUDA tensor, learnable, or a number) is shared by all pairs and levels;
    each level runs `iters` sweeps, checkpointed every `ckpt_every` for the reverse mode.
    All pairs of a level go through one batched Horn-Schunck call.
    """
    if levels < 1:
        raise ValueError("levels must be >= 1")
    n = len(pairs)
    if n < 1 or n > L.HS_MAX_TRAIN_PAIRS:
        raise ValueError(f"1..{L.HS_MAX_TRAIN_PAIRS} pairs, got {n}")
    dev = pairs[0][0].device
    if not isinstance(alpha, torch.Tensor):
        alpha = torch.tensor(float(alpha), dtype=torch.float32, device=dev)
    p0 = [build_pyramid(a, levels) for a, _ in pairs]
    p1 = [build_pyramid(b, levels) for _, b in pairs]
    flows = None
    for lev in range(levels - 1, -1, -1):
        if flows is None:
            lvl_pairs = [(p0[i][lev], p1[i][lev]) for i in range(n)]
        else:
            up = []
            for i in range(n):
                H, W = p0[i][lev].shape
                up.append((upsample2(flows[i][0], H, W), upsample2(flows[i][1], H, W)))
            lvl_pairs = [(p0[i][lev], warp(p1[i][lev], up[i][0], up[i][1])) for i in range(n)]
        inc = horn_schunck_batch(lvl_pairs, alpha, iters, ckpt_every, config)
        if flows is None:
            flows = inc
        else:
            flows = [(up[i][0] + inc[i][0], up[i][1] + inc[i][1]) for i in range(n)]
    return flows
