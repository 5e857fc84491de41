"""Lucas-Kanade and the Brox solver's building blocks on the device (libhsflow kernels):
``lk_least_squares`` (LKLeastSquares), ``set_brox_matrix`` / ``set_brox_redblack_matrix``
(SetBroxMatrix / SetBroxRedblackMatrix), ``spmv_dia2d`` (SpmvDIA2D) and
``apply_brox_preconditioner`` (ApplyBroxPreconditioner).  A ``DeviceSpMat2D`` keeps the
diagonals of a grid operator as one (ndiags, H, ld) float32 CUDA tensor.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np
import torch

from . import _lib as L
from . import device as D


class DeviceSpMat2D:
    def __init__(self, data: torch.Tensor, offx, offy, W: int):
        self.buf = data                    # (ndiags, H, ld)
        self.offx = np.ascontiguousarray(offx, dtype=np.int32)
        self.offy = np.ascontiguousarray(offy, dtype=np.int32)
        self.ndiags, self.H, self.ld = data.shape
        self.W = W

    @classmethod
    def from_host(cls, A, device=None) -> "DeviceSpMat2D":
        """Copy an SpMat2D (NumPy or torch data of shape (ndiags, H, W)) to the device."""
        data = A.data
        if isinstance(data, np.ndarray):
            data = torch.from_numpy(np.ascontiguousarray(data, dtype=np.float32))
        n, H, W = data.shape
        buf = torch.zeros((n, H, D.padded_ld(W)), dtype=torch.float32, device=device or "cuda")
        buf[:, :, :W].copy_(data)
        return cls(buf, A.offx, A.offy, W)

    @property
    def diag_stride(self) -> int:
        return self.H * self.ld

    def diagonal(self, d: int) -> torch.Tensor:
        return self.buf[d, :, :self.W]

    def data(self) -> torch.Tensor:
        return self.buf[:, :, :self.W]


def _plane_ld(t: torch.Tensor, ld: int) -> torch.Tensor:
    if D.is_plane(t) and t.stride(0) == ld:
        return t
    H, W = t.shape
    p = torch.empty((H, ld), dtype=torch.float32, device=t.device)[:, :W]
    p.copy_(t)
    return p


def lk_least_squares(err, Ix, Iy, radius: int) -> Tuple[torch.Tensor, torch.Tensor]:
    err, Ix, Iy = D._same_layout(err, Ix, Iy)
    H, W = err.shape
    out = torch.empty((2, H, err.stride(0)), dtype=torch.float32, device=err.device)[:, :, :W]
    L.check(L.lib().hs_lk_least_squares(D.ptr(err), D.ptr(Ix), D.ptr(Iy), H, W, err.stride(0),
                                        int(radius), D.ptr(out[0]), D.ptr(out[1]),
                                        D.stream_handle()), "hs_lk_least_squares")
    return out[0], out[1]


def set_brox_matrix(A: DeviceSpMat2D, psi, alpha: float) -> None:
    """Fill A's 5 diagonals (top, left, mid, right, bottom) in place."""
    if A.ndiags != 5:
        raise ValueError("set_brox_matrix needs a 5-diagonal SpMat2D")
    psi = _plane_ld(D.as_plane(psi), A.ld)
    L.check(L.lib().hs_set_brox_matrix(D.ptr(psi), A.H, A.W, A.ld, float(np.float32(alpha)),
                                       D.ptr(A.buf), A.diag_stride, 0, None, D.stream_handle()),
            "hs_set_brox_matrix")


def set_brox_redblack_matrix(A: DeviceSpMat2D, psi, alpha: float) -> torch.Tensor:
    """Fill A's 4 off-diagonals (top, left, right, bottom) in place; returns the middle term."""
    if A.ndiags != 4:
        raise ValueError("set_brox_redblack_matrix needs a 4-diagonal SpMat2D")
    psi = _plane_ld(D.as_plane(psi), A.ld)
    adiag = torch.empty((A.H, A.ld), dtype=torch.float32, device=A.buf.device)[:, :A.W]
    L.check(L.lib().hs_set_brox_matrix(D.ptr(psi), A.H, A.W, A.ld, float(np.float32(alpha)),
                                       D.ptr(A.buf), A.diag_stride, 1, D.ptr(adiag),
                                       D.stream_handle()), "hs_set_brox_matrix")
    return adiag


def spmv_dia2d(A: DeviceSpMat2D, x) -> torch.Tensor:
    x = _plane_ld(D.as_plane(x), A.ld)
    if x.shape != (A.H, A.W):
        raise ValueError(f"SpMat2D {A.H}x{A.W} times an array of shape {tuple(x.shape)}")
    y = torch.empty((A.H, A.ld), dtype=torch.float32, device=x.device)[:, :A.W]
    L.check(L.lib().hs_spmv_dia2d(D.ptr(A.buf), A.diag_stride, A.offx.ctypes.data_as(L._ip),
                                  A.offy.ctypes.data_as(L._ip), A.ndiags, D.ptr(x), A.H, A.W, A.ld,
                                  D.ptr(y), D.stream_handle()), "hs_spmv_dia2d")
    return y


def apply_brox_preconditioner(A: DeviceSpMat2D, diag0, diag1, offdiag, x0, x1):
    """The reference's applyBroxPreconditioner(D, diag0, diag1, offdiag, x0, x1): the middle
    diagonal of D (diagonal 2) enters the 2x2 blocks."""
    planes = [_plane_ld(D.as_plane(t), A.ld) for t in (diag0, diag1, offdiag, x0, x1)]
    y = torch.empty((2, A.H, A.ld), dtype=torch.float32, device=planes[0].device)[:, :, :A.W]
    L.check(L.lib().hs_apply_brox_preconditioner(D.ptr(A.diagonal(2)), *(D.ptr(p) for p in planes),
                                                 A.H, A.W, A.ld, D.ptr(y[0]), D.ptr(y[1]),
                                                 D.stream_handle()), "hs_apply_brox_preconditioner")
    return y[0], y[1]
