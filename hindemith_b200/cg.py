"""Horn-Schunck as a linear system: the operator's Krylov powers (``hs_matrix_powers``,
the reference's HSMatrixPowers) and the 2x2 block-Jacobi preconditioner
(``apply_hs_preconditioner``, ApplyHSPreconditioner), both libhsflow kernels, plus a
preconditioned conjugate-gradient solver built from them.

The HS Euler-Lagrange equations are M w = b with
    M (u, v) = (Ix (Ix u + Iy v), Iy (Ix u + Iy v)) + lam * L (u, v),  lam = alpha^2,
L the 4-neighbour graph Laplacian with no flux across the border, and b = -(Ix It, Iy It).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import torch

from . import _lib as L
from . import device as D


def hs_matrix_powers(lam: float, Ix, Iy, r0, r1, steps: int,
                     config: Optional[L.hs_config] = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """V0, V1 of shape (steps, H, W): V[0] = (r0, r1), V[s] = M V[s-1]."""
    Ix, Iy, r0, r1 = D._same_layout(Ix, Iy, r0, r1)
    H, W = Ix.shape
    ld = Ix.stride(0)
    if steps < 1:
        raise ValueError("steps must be >= 1")
    buf = torch.empty((2, steps, H, ld), dtype=torch.float32, device=Ix.device)
    cfg = config if config is not None else L.make_config()
    L.check(L.lib().hs_matrix_powers(float(lam), D.ptr(Ix), D.ptr(Iy), D.ptr(r0), D.ptr(r1), H, W,
                                     ld, int(steps), D.ptr(buf[0]), D.ptr(buf[1]), H * ld,
                                     ctypes.byref(cfg), D.stream_handle()), "hs_matrix_powers")
    return buf[0, :, :, :W], buf[1, :, :, :W]


def _stencil_s2(Dst) -> float:
    data = getattr(Dst, "data", None)
    if data is not None:
        return float(data[2])
    return float(Dst)


def apply_hs_preconditioner(Dst, diag0, diag1, offdiag, x0, x1) -> Tuple[torch.Tensor, torch.Tensor]:
    """The reference's applyHSPreconditioner(D, diag0, diag1, offdiag, x0, x1); D is a
    Stencil (its third weight is used) or that weight as a number."""
    diag0, diag1, offdiag, x0, x1 = D._same_layout(diag0, diag1, offdiag, x0, x1)
    H, W = x0.shape
    y = torch.empty((2, H, x0.stride(0)), dtype=torch.float32, device=x0.device)[:, :, :W]
    L.check(L.lib().hs_apply_hs_preconditioner(_stencil_s2(Dst), D.ptr(diag0), D.ptr(diag1),
                                               D.ptr(offdiag), D.ptr(x0), D.ptr(x1), H, W,
                                               x0.stride(0), D.ptr(y[0]), D.ptr(y[1]),
                                               D.stream_handle()), "hs_apply_hs_preconditioner")
    return y[0], y[1]


def hs_pcg(Ix, Iy, It, alpha: float, iters: int, tol: float = 0.0):
    """Solve the HS system M w = -(Ix It, Iy It), lam = alpha^2, by conjugate gradients
    preconditioned with the 2x2 block Jacobi step.  The operator and the preconditioner
    run as libhsflow kernels; the inner products accumulate in float64.  Returns (u, v,
    relative residual norms per iteration)."""
    Ix, Iy, It = D._same_layout(Ix, Iy, It)
    lam = float(alpha) * float(alpha)
    bu, bv = -(Ix * It), -(Iy * It)
    d0, d1, od = Ix * Ix, Iy * Iy, Ix * Iy
    u = torch.zeros_like(bu)
    v = torch.zeros_like(bv)
    ru, rv = bu.clone(), bv.clone()

    def dot(a0, a1, b0, b1):
        return (a0.double() * b0.double()).sum() + (a1.double() * b1.double()).sum()

    bnorm = torch.sqrt(dot(bu, bv, bu, bv)).clamp_min(1e-300)
    zu, zv = apply_hs_preconditioner(lam, d0, d1, od, ru, rv)
    pu, pv = zu.clone(), zv.clone()
    rz = dot(ru, rv, zu, zv)
    hist = []
    for _ in range(int(iters)):
        V0, V1 = hs_matrix_powers(lam, Ix, Iy, pu, pv, 2)
        qu, qv = V0[1], V1[1]
        a = (rz / dot(pu, pv, qu, qv)).float()
        u = u + a * pu
        v = v + a * pv
        ru = ru - a * qu
        rv = rv - a * qv
        hist.append(torch.sqrt(dot(ru, rv, ru, rv)) / bnorm)
        zu, zv = apply_hs_preconditioner(lam, d0, d1, od, ru, rv)
        rz_new = dot(ru, rv, zu, zv)
        beta = (rz_new / rz).float()
        rz = rz_new
        pu = zu + beta * pu
        pv = zv + beta * pv
    res = torch.stack(hist).cpu() if hist else torch.zeros(0, dtype=torch.float64)
    if tol > 0 and len(res) and float(res[-1]) > tol:
        raise RuntimeError(f"hs_pcg: relative residual {float(res[-1]):.3e} above {tol:.1e}")
    return u, v, res
