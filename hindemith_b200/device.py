"""Torch-tensor front of libhsflow: device planes, workspaces, streams.

PyTorch supplies device memory and the current CUDA stream; every computation is a
libhsflow kernel reached through the C ABI.  A *plane* is a 2-D float32 CUDA tensor
of shape (H, W) whose row stride (the ABI's ``ld``) is a multiple of 4 elements and
whose storage starts on a 16-byte boundary; ``as_plane`` copies anything else into
such a layout.
"""
from __future__ import annotations

import contextlib
import ctypes
import functools
import inspect
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib as L


def _require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (libhsflow has no CPU path)")


def on_stream(fn):
    """Run `fn` with its `stream` argument (when given) as torch's current stream.

    Every tensor the call allocates -- outputs, copied inputs, cached scratch -- then
    belongs to the stream its kernels run on, so the caching allocator never hands that
    memory to another stream while those kernels may still use it."""
    pos = list(inspect.signature(fn).parameters).index("stream")

    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        s = kwargs.get("stream", args[pos] if len(args) > pos else None)
        if s is None:
            return fn(*args, **kwargs)
        with torch.cuda.stream(s):
            return fn(*args, **kwargs)

    return wrapper


def stream_scope(stream=None):
    """Context making `stream` (when given) torch's current stream."""
    return contextlib.nullcontext() if stream is None else torch.cuda.stream(stream)


def stream_handle(stream: Optional[torch.cuda.Stream] = None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def padded_ld(W: int) -> int:
    return (W + 3) // 4 * 4


def empty_planes(n: int, H: int, W: int, device=None) -> torch.Tensor:
    """n planes (n, H, W) sharing one allocation, each row padded to a multiple of 4."""
    ld = padded_ld(W)
    buf = torch.empty((n, H, ld), dtype=torch.float32, device=device or "cuda")
    return buf[:, :, :W]


def empty_plane(H: int, W: int, device=None) -> torch.Tensor:
    return empty_planes(1, H, W, device)[0]


def zeros_plane(H: int, W: int, device=None) -> torch.Tensor:
    p = empty_plane(H, W, device)
    p.zero_()
    return p


def is_plane(t: torch.Tensor) -> bool:
    return (t.dim() == 2 and t.dtype == torch.float32 and t.is_cuda and t.stride(1) == 1
            and t.stride(0) % 4 == 0 and t.stride(0) >= t.shape[1] and t.data_ptr() % 16 == 0)


def as_plane(x, device=None) -> torch.Tensor:
    """Return `x` as a plane (no copy when it already is one)."""
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32))
    if not isinstance(x, torch.Tensor):
        raise TypeError(f"expected a 2-D array, got {type(x).__name__}")
    if x.dim() != 2:
        raise ValueError(f"expected a 2-D array, got shape {tuple(x.shape)}")
    if is_plane(x):
        return x
    dev = device or (x.device if x.is_cuda else "cuda")
    p = empty_plane(x.shape[0], x.shape[1], dev)
    p.copy_(x.to(torch.float32), non_blocking=True)
    return p


def ld_of(p: torch.Tensor) -> int:
    return p.stride(0)


def ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


# ------------------------------------------------------------------ workspaces

_workspaces = {}


def workspace(nbytes: int, device: torch.device, stream=None) -> torch.Tensor:
    """A cached scratch buffer of at least `nbytes` bytes for (device, stream).

    Calls issued on one stream run in order, so they may share its buffer; distinct
    streams get distinct buffers.  The buffer is allocated on that stream, so when a
    larger one replaces it the allocator reuses the old memory only in that stream's
    order.
    """
    s = stream if stream is not None else torch.cuda.current_stream(device)
    key = (torch.device(device).index, s.cuda_stream)
    buf = _workspaces.get(key)
    if buf is None or buf.numel() < nbytes:
        with torch.cuda.stream(s):
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _workspaces[key] = buf
    return buf


def release_workspaces() -> None:
    _workspaces.clear()


# ------------------------------------------------------------------ operations


@on_stream
def stencil2d(weights, offx, offy, x: torch.Tensor, out: Optional[torch.Tensor] = None,
              stream=None) -> torch.Tensor:
    """out = S * x for the clamp-to-edge stencil S (Stencil2DMVM)."""
    x = as_plane(x)
    H, W = x.shape
    w = np.ascontiguousarray(weights, dtype=np.float32)
    ox = np.ascontiguousarray(offx, dtype=np.int32)
    oy = np.ascontiguousarray(offy, dtype=np.int32)
    if not (len(w) == len(ox) == len(oy)):
        raise ValueError("stencil data, offx and offy must have the same length")
    if out is None:
        out = _like(x)
    elif not is_plane(out) or out.shape != x.shape:
        raise ValueError("out must be a plane of the input's shape")
    st = L.lib().hs_stencil2d(w.ctypes.data_as(L._fp), ox.ctypes.data_as(L._ip),
                              oy.ctypes.data_as(L._ip), len(w), ptr(x), ptr(out), H, W,
                              ld_of(x), stream_handle(stream))
    L.check(st, "hs_stencil2d")
    return out


def _like(x: torch.Tensor) -> torch.Tensor:
    H, W = x.shape
    return torch.empty((H, x.stride(0)), dtype=torch.float32, device=x.device)[:, :W]


def _same_layout(*ts) -> Tuple[torch.Tensor, ...]:
    """Planes sharing one ld (the pointwise ABI takes a single ld)."""
    planes = [as_plane(t) for t in ts]
    ld = planes[0].stride(0)
    out = []
    for p in planes:
        if p.stride(0) != ld:
            q = torch.empty((p.shape[0], ld), dtype=torch.float32, device=p.device)[:, :p.shape[1]]
            q.copy_(p)
            p = q
        out.append(p)
    return tuple(out)


@on_stream
def array2d_op(op: int, b, c, stream=None) -> torch.Tensor:
    b, c = _same_layout(b, c)
    if b.shape != c.shape:
        raise ValueError(f"shape mismatch {tuple(b.shape)} vs {tuple(c.shape)}")
    a = _like(b)
    H, W = b.shape
    L.check(L.lib().hs_array2d_op(op, ptr(b), ptr(c), ptr(a), H, W, ld_of(b),
                                  stream_handle(stream)), "hs_array2d_op")
    return a


@on_stream
def array2d_scalar_op(op: int, b, s: float, stream=None) -> torch.Tensor:
    b = as_plane(b)
    a = _like(b)
    H, W = b.shape
    L.check(L.lib().hs_array2d_scalar_op(op, ptr(b), float(np.float32(s)), ptr(a), H, W,
                                         ld_of(b), stream_handle(stream)), "hs_array2d_scalar_op")
    return a


@on_stream
def scalar_array2d_op(op: int, s: float, b, stream=None) -> torch.Tensor:
    b = as_plane(b)
    a = _like(b)
    H, W = b.shape
    L.check(L.lib().hs_scalar_array2d_op(op, float(np.float32(s)), ptr(b), ptr(a), H, W,
                                         ld_of(b), stream_handle(stream)), "hs_scalar_array2d_op")
    return a


@on_stream
def array2d_copy(b, stream=None) -> torch.Tensor:
    b = as_plane(b)
    a = _like(b)
    H, W = b.shape
    L.check(L.lib().hs_array2d_copy(ptr(b), ptr(a), H, W, ld_of(b), stream_handle(stream)),
            "hs_array2d_copy")
    return a


@on_stream
def hs_derivs(I0, I1, stream=None):
    """(Ix, Iy, It) of the 2x2x2 Horn-Schunck derivatives, one fused pass."""
    I0, I1 = _same_layout(I0, I1)
    if I0.shape != I1.shape:
        raise ValueError("I0 and I1 must have the same shape")
    H, W = I0.shape
    out = torch.empty((3, H, I0.stride(0)), dtype=torch.float32, device=I0.device)[:, :, :W]
    Ix, Iy, It = out[0], out[1], out[2]
    L.check(L.lib().hs_derivs(ptr(I0), ptr(I1), H, W, ld_of(I0), ptr(Ix), ptr(Iy), ptr(It),
                              stream_handle(stream)), "hs_derivs")
    return Ix, Iy, It


@on_stream
def hs_sweeps(Ix, Iy, It, alpha2: float, iters: int, u: torch.Tensor, v: torch.Tensor,
              config: Optional[L.hs_config] = None, stream=None) -> None:
    """`iters` Jacobi sweeps in place on the planes u, v (same layout as Ix)."""
    Ix, Iy, It = _same_layout(Ix, Iy, It)
    for name, t in (("u", u), ("v", v)):
        if not is_plane(t) or t.stride(0) != Ix.stride(0) or t.shape != Ix.shape:
            raise ValueError(f"{name} must be a plane with the layout of Ix")
    H, W = Ix.shape
    ld = ld_of(Ix)
    nbytes = L.lib().hs_sweeps_workspace_bytes(H, W, ld)
    ws = workspace(nbytes, Ix.device, stream)
    cfg = config if config is not None else L.make_config()
    L.check(L.lib().hs_sweeps(ptr(Ix), ptr(Iy), ptr(It), H, W, ld, float(np.float32(alpha2)),
                              int(iters), ptr(u), ptr(v), ptr(ws), ws.numel(),
                              ctypes.byref(cfg), stream_handle(stream)), "hs_sweeps")


@on_stream
def hs_forward(I0, I1, alpha: float, iters: int, config: Optional[L.hs_config] = None,
               stream=None, out=None):
    """Plain per-pair Horn-Schunck: derivatives, u = v = 0, `iters` sweeps.

    Returns (u, v) planes.  `out` may supply a (2, H, ld)-backed pair to write into.
    """
    I0, I1 = _same_layout(I0, I1)
    if I0.shape != I1.shape:
        raise ValueError("I0 and I1 must have the same shape")
    H, W = I0.shape
    ld = ld_of(I0)
    if out is None:
        uv = torch.empty((2, H, ld), dtype=torch.float32, device=I0.device)[:, :, :W]
        u, v = uv[0], uv[1]
    else:
        u, v = out
    nbytes = L.lib().hs_forward_workspace_bytes(H, W, ld)
    ws = workspace(nbytes, I0.device, stream)
    cfg = config if config is not None else L.make_config()
    L.check(L.lib().hs_forward(ptr(I0), ptr(I1), H, W, ld, float(np.float32(alpha)), int(iters),
                               ptr(u), ptr(v), ptr(ws), ws.numel(), ctypes.byref(cfg),
                               stream_handle(stream)), "hs_forward")
    return u, v


@on_stream
def warp(src, u, v, stream=None) -> torch.Tensor:
    """WarpImg2D: src backward-warped by (u, v) (Operations/OpticalFlow/WarpImg2D.cpp:33-75)."""
    src, u, v = _same_layout(src, u, v)
    if u.shape != src.shape or v.shape != src.shape:
        raise ValueError("warp_img2d needs src, u and v of one shape")
    out = _like(src)
    H, W = src.shape
    L.check(L.lib().hs_warp(ptr(src), ptr(u), ptr(v), H, W, ld_of(src), ptr(out),
                            stream_handle(stream)), "hs_warp")
    return out
