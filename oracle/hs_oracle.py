"""CPU oracle for the Horn-Schunck stencil path (TEST INFRASTRUCTURE ONLY).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use this module, always as the checker.  The product package never imports it.

Two restatements of the reference's semantics live here:

* NumPy functions (``stencil2d``, ``hs_derivs``, ``hs_sweeps``, ``hs_forward``,
  ``warp``).  With ``dtype=np.float32`` they do one IEEE-rounded FP32 operation at a
  time, in the order the reference program performs them, so they match the
  reference's FP32 results bit for bit.  With ``dtype=np.float64`` they are the
  accuracy reference.
* ctypes wrappers (``c_*``) over ``oracle/hs_oracle.c``, the same restatement in C
  with OpenMP, fast enough for full-size checks and the CPU baseline.

Reference anchors (paths inside chick/hindemith):
  Stencil2DMVM.cpp:34-59      clamp-to-edge tap loop, accumulate from 0 in tap order
  Types/Array2D.cpp:302,333   element index x + y*W (x = last NumPy axis)
  Array2DOp.cpp:27-53         a = b op c, op in {+,-,*,/}
  Array2DScalarOp.cpp:29-55   a = b op *scalar
  ScalarArray2DOp.cpp:29-55   a = *scalar op b
  WarpImg2D.cpp:33-75         bilinear backward warp, source pixel when out of bounds
  hlib.py:173-191             NumPy Stencil.__mul__ (edge padding; symmetric stencils)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhsoracle.so")

# Canonical Horn-Schunck stencils, tap order (offx, offy).  Identical tables live in the
# CUDA sources and in hindemith_b200.hlib; the tests check that they agree.
AVG_OFFX = np.array([-1, 0, 1, -1, 1, -1, 0, 1], dtype=np.int32)
AVG_OFFY = np.array([-1, -1, -1, 0, 0, 1, 1, 1], dtype=np.int32)
AVG_W = np.array([1 / 12 if (ox != 0 and oy != 0) else 1 / 6
                  for ox, oy in zip(AVG_OFFX, AVG_OFFY)], dtype=np.float32)
D_OFFX = np.array([0, 1, 0, 1], dtype=np.int32)
D_OFFY = np.array([0, 0, 1, 1], dtype=np.int32)
DX_W = np.array([-0.25, 0.25, -0.25, 0.25], dtype=np.float32)
DY_W = np.array([-0.25, -0.25, 0.25, 0.25], dtype=np.float32)
DT_W = np.array([0.25, 0.25, 0.25, 0.25], dtype=np.float32)


# ---------------------------------------------------------------- NumPy restatement

def stencil2d(w, offx, offy, x, dtype=np.float32):
    """y[r, c] = sum_d w[d] * x[clamp(r + offy[d]), clamp(c + offx[d])], from 0, tap order.

    Stencil2DMVM.cpp:37-48.  Each product and each sum rounds to ``dtype``.
    """
    x = np.asarray(x, dtype=dtype)
    H, W = x.shape
    rows = np.arange(H)
    cols = np.arange(W)
    acc = np.zeros((H, W), dtype=dtype)
    for d in range(len(w)):
        rr = np.clip(rows + int(offy[d]), 0, H - 1)
        cc = np.clip(cols + int(offx[d]), 0, W - 1)
        acc = acc + dtype(w[d]) * x[rr][:, cc]
    return acc


def stencil2d_transpose(w, offx, offy, x, dtype=np.float64):
    """S^T x for the clamp-to-edge stencil S (scatter form; small sizes only)."""
    x = np.asarray(x, dtype=dtype)
    H, W = x.shape
    out = np.zeros((H, W), dtype=dtype)
    rows = np.arange(H)
    cols = np.arange(W)
    for d in range(len(w)):
        rr = np.clip(rows + int(offy[d]), 0, H - 1)
        cc = np.clip(cols + int(offx[d]), 0, W - 1)
        np.add.at(out, (rr[:, None], cc[None, :]), dtype(w[d]) * x)
    return out


def hs_derivs(I0, I1, dtype=np.float32):
    """Ix = Dx*I0 + Dx*I1, Iy = Dy*I0 + Dy*I1, It = Dt*I1 - Dt*I0."""
    Ix = stencil2d(DX_W, D_OFFX, D_OFFY, I0, dtype) + stencil2d(DX_W, D_OFFX, D_OFFY, I1, dtype)
    Iy = stencil2d(DY_W, D_OFFX, D_OFFY, I0, dtype) + stencil2d(DY_W, D_OFFX, D_OFFY, I1, dtype)
    It = stencil2d(DT_W, D_OFFX, D_OFFY, I1, dtype) - stencil2d(DT_W, D_OFFX, D_OFFY, I0, dtype)
    return Ix, Iy, It


def hs_sweeps(Ix, Iy, It, alpha2, iters, u, v, dtype=np.float32):
    """`iters` Jacobi sweeps: ubar = A*u; vbar = A*v;
    t = (Ix*ubar + Iy*vbar + It) / (alpha2 + Ix*Ix + Iy*Iy); u = ubar - Ix*t; v = vbar - Iy*t.
    """
    Ix, Iy, It = (np.asarray(a, dtype=dtype) for a in (Ix, Iy, It))
    u = np.array(u, dtype=dtype)
    v = np.array(v, dtype=dtype)
    a2 = dtype(alpha2)
    den = a2 + Ix * Ix + Iy * Iy
    for _ in range(iters):
        ubar = stencil2d(AVG_W, AVG_OFFX, AVG_OFFY, u, dtype)
        vbar = stencil2d(AVG_W, AVG_OFFX, AVG_OFFY, v, dtype)
        t = (Ix * ubar + Iy * vbar + It) / den
        u = ubar - Ix * t
        v = vbar - Iy * t
    return u, v


def hs_forward(I0, I1, alpha, iters, dtype=np.float32):
    """Derivatives, u = v = 0, `iters` sweeps; alpha2 = alpha * alpha in ``dtype``."""
    Ix, Iy, It = hs_derivs(I0, I1, dtype)
    z = np.zeros(np.shape(I0), dtype=dtype)
    a = dtype(alpha)
    return hs_sweeps(Ix, Iy, It, a * a, iters, z, z, dtype)


def warp(src, ox, oy):
    """WarpImg2D.cpp:33-75 with its FP32/FP64 roundings (see hs_oracle.c)."""
    src = np.asarray(src, dtype=np.float32)
    ox = np.asarray(ox, dtype=np.float32)
    oy = np.asarray(oy, dtype=np.float32)
    H, W = src.shape
    mx = np.trunc(ox).astype(np.int64)
    my = np.trunc(oy).astype(np.int64)
    xf = (ox - mx.astype(np.float32)).astype(np.float32)
    yf = (oy - my.astype(np.float32)).astype(np.float32)
    negx = ox < 0
    negy = oy < 0
    mx = np.where(negx, mx - 1, mx)
    my = np.where(negy, my - 1, my)
    xf = np.where(negx, (1.0 + xf.astype(np.float64)).astype(np.float32), xf)
    yf = np.where(negy, (1.0 + yf.astype(np.float64)).astype(np.float32), yf)
    X, Y = np.meshgrid(np.arange(W), np.arange(H))
    ok = (X + mx >= 0) & (X + mx + 1 < W) & (Y + my >= 0) & (Y + my + 1 < H)
    bx = np.where(ok, X + mx, 0)
    by = np.where(ok, Y + my, 0)
    bx1 = np.minimum(bx + 1, W - 1)
    by1 = np.minimum(by + 1, H - 1)
    xd = xf.astype(np.float64)
    yd = yf.astype(np.float64)
    s = src.astype(np.float64)
    # C's typing of the template's expressions, left to right: float products until
    # (1.0 - frac) makes them double
    o = np.zeros((H, W), dtype=np.float32)
    o = (o + s[by, bx] * (1.0 - xd) * (1.0 - yd)).astype(np.float32)
    o = (o + (src[by, bx1] * xf).astype(np.float64) * (1.0 - yd)).astype(np.float32)
    o = (o + s[by1, bx] * (1.0 - xd) * yd).astype(np.float32)
    o = o + (src[by1, bx1] * xf) * yf
    return np.where(ok, o, src).astype(np.float32)


# ---------------------------------------------------------------- C restatement

_lib = None


def build():
    """Compile hs_oracle.c into oracle/_build/libhsoracle.so."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        c_int, c_float, c_double = ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.hso_num_threads.restype = c_int
        L.hso_set_num_threads.argtypes = [c_int]
        L.hso_stencil2d_f32.argtypes = [f32p, i32p, i32p, c_int, f32p, f32p, c_int, c_int]
        L.hso_stencil2d_f64.argtypes = [f64p, i32p, i32p, c_int, f64p, f64p, c_int, c_int]
        L.hso_stencil2d_transpose_f64.argtypes = [f64p, i32p, i32p, c_int, f64p, f64p, c_int, c_int]
        L.hso_hs_derivs_f32.argtypes = [f32p, f32p, c_int, c_int, f32p, f32p, f32p]
        L.hso_hs_derivs_f64.argtypes = [f64p, f64p, c_int, c_int, f64p, f64p, f64p]
        L.hso_hs_sweeps_f32.argtypes = [f32p, f32p, f32p, c_int, c_int, c_float, c_int, f32p, f32p]
        L.hso_hs_sweeps_f64.argtypes = [f64p, f64p, f64p, c_int, c_int, c_double, c_int, f64p, f64p]
        L.hso_hs_forward_f32.argtypes = [f32p, f32p, c_int, c_int, c_float, c_int, f32p, f32p]
        L.hso_hs_forward_f64.argtypes = [f64p, f64p, c_int, c_int, c_double, c_int, f64p, f64p]
        L.hso_warp_f32.argtypes = [f32p, f32p, f32p, c_int, c_int, f32p]
        L.hso_hs_matrix_powers_f32.argtypes = [c_float, f32p, f32p, f32p, f32p, c_int, c_int,
                                               c_int, f32p, f32p]
        L.hso_apply_hs_precond_f32.argtypes = [c_float, f32p, f32p, f32p, f32p, f32p, c_int,
                                               c_int, f32p, f32p]
        L.hso_lk_least_squares_f32.argtypes = [f32p, f32p, f32p, c_int, c_int, c_int, f32p, f32p]
        L.hso_set_brox_matrix_f32.argtypes = [f32p, c_int, c_int, c_float, f32p, c_int, f32p]
        L.hso_spmv_dia2d_f32.argtypes = [f32p, i32p, i32p, c_int, f32p, c_int, c_int, f32p]
        L.hso_apply_brox_precond_f32.argtypes = [f32p, f32p, f32p, f32p, f32p, f32p, c_int, c_int,
                                                 f32p, f32p]
        for name in ("hso_hs_sweeps_f32", "hso_hs_sweeps_f64", "hso_hs_forward_f32",
                     "hso_hs_forward_f64"):
            getattr(L, name).restype = c_int
        _lib = L
    return _lib


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def c_num_threads():
    return lib().hso_num_threads()


def c_set_num_threads(n):
    """OpenMP threads of the C restatement's loops from now on (n >= 1)."""
    lib().hso_set_num_threads(int(n))


def c_stencil2d(w, offx, offy, x, dtype=np.float32):
    x = np.ascontiguousarray(x, dtype=dtype)
    H, W = x.shape
    out = np.empty_like(x)
    ox = np.ascontiguousarray(offx, dtype=np.int32)
    oy = np.ascontiguousarray(offy, dtype=np.int32)
    if dtype == np.float32:
        lib().hso_stencil2d_f32(_c32(w), ox, oy, len(ox), x, out, H, W)
    else:
        lib().hso_stencil2d_f64(_c64(w), ox, oy, len(ox), x, out, H, W)
    return out


def c_stencil2d_transpose(w, offx, offy, x):
    x = _c64(x)
    H, W = x.shape
    out = np.empty_like(x)
    ox = np.ascontiguousarray(offx, dtype=np.int32)
    oy = np.ascontiguousarray(offy, dtype=np.int32)
    lib().hso_stencil2d_transpose_f64(_c64(w), ox, oy, len(ox), x, out, H, W)
    return out


def c_hs_derivs(I0, I1, dtype=np.float32):
    conv = _c32 if dtype == np.float32 else _c64
    I0, I1 = conv(I0), conv(I1)
    H, W = I0.shape
    Ix, Iy, It = (np.empty_like(I0) for _ in range(3))
    fn = lib().hso_hs_derivs_f32 if dtype == np.float32 else lib().hso_hs_derivs_f64
    fn(I0, I1, H, W, Ix, Iy, It)
    return Ix, Iy, It


def c_hs_sweeps(Ix, Iy, It, alpha2, iters, u, v, dtype=np.float32):
    conv = _c32 if dtype == np.float32 else _c64
    Ix, Iy, It = conv(Ix), conv(Iy), conv(It)
    u = conv(u).copy()
    v = conv(v).copy()
    H, W = Ix.shape
    fn = lib().hso_hs_sweeps_f32 if dtype == np.float32 else lib().hso_hs_sweeps_f64
    if fn(Ix, Iy, It, H, W, alpha2, int(iters), u, v) != 0:
        raise MemoryError("oracle sweep allocation failed")
    return u, v


def c_hs_forward(I0, I1, alpha, iters, dtype=np.float32):
    conv = _c32 if dtype == np.float32 else _c64
    I0, I1 = conv(I0), conv(I1)
    H, W = I0.shape
    u = np.empty_like(I0)
    v = np.empty_like(I0)
    fn = lib().hso_hs_forward_f32 if dtype == np.float32 else lib().hso_hs_forward_f64
    if fn(I0, I1, H, W, alpha, int(iters), u, v) != 0:
        raise MemoryError("oracle forward allocation failed")
    return u, v


def c_warp(src, ox, oy):
    src, ox, oy = _c32(src), _c32(ox), _c32(oy)
    H, W = src.shape
    out = np.empty_like(src)
    lib().hso_warp_f32(src, ox, oy, H, W, out)
    return out


def c_hs_matrix_powers(lam, Ix, Iy, r0, r1, steps):
    """HSMatrixPowers.cpp:72-106 in FP32, template operation order -> V0, V1 (steps, H, W)."""
    Ix, Iy, r0, r1 = _c32(Ix), _c32(Iy), _c32(r0), _c32(r1)
    H, W = Ix.shape
    V0 = np.empty((steps, H, W), np.float32)
    V1 = np.empty((steps, H, W), np.float32)
    lib().hso_hs_matrix_powers_f32(float(np.float32(lam)), Ix, Iy, r0, r1, H, W, int(steps), V0, V1)
    return V0, V1


def c_apply_hs_precond(s2, diag0, diag1, offdiag, x0, x1):
    """ApplyHSPreconditioner.cpp:46-97 in FP32 -> y0, y1."""
    diag0, diag1, offdiag, x0, x1 = (_c32(a) for a in (diag0, diag1, offdiag, x0, x1))
    H, W = x0.shape
    y0, y1 = np.empty_like(x0), np.empty_like(x0)
    lib().hso_apply_hs_precond_f32(float(np.float32(s2)), diag0, diag1, offdiag, x0, x1, H, W, y0, y1)
    return y0, y1


def c_lk_least_squares(err, Ix, Iy, rad):
    """LKLeastSquares.cpp:44-79 in FP32 -> du, dv."""
    err, Ix, Iy = _c32(err), _c32(Ix), _c32(Iy)
    H, W = err.shape
    du, dv = np.empty_like(err), np.empty_like(err)
    lib().hso_lk_least_squares_f32(err, Ix, Iy, H, W, int(rad), du, dv)
    return du, dv


def c_set_brox_matrix(psi, alpha, data, redblack=False):
    """SetBroxMatrix.cpp / SetBroxRedblackMatrix.cpp in FP32: updates a copy of `data`
    (ndiags, H, W) and returns it (and the mid term for the red-black form)."""
    psi = _c32(psi)
    H, W = psi.shape
    data = _c32(data).copy()
    adiag = np.zeros((H, W), np.float32)
    lib().hso_set_brox_matrix_f32(psi, H, W, float(np.float32(alpha)), data, 1 if redblack else 0, adiag)
    return (data, adiag) if redblack else data


def c_spmv_dia2d(data, offx, offy, x):
    """SpmvDIA2D.cpp:36-45 in FP32."""
    data, x = _c32(data), _c32(x)
    H, W = x.shape
    out = np.empty_like(x)
    ox = np.ascontiguousarray(offx, dtype=np.int32)
    oy = np.ascontiguousarray(offy, dtype=np.int32)
    lib().hso_spmv_dia2d_f32(data, ox, oy, len(ox), x, H, W, out)
    return out


def c_apply_brox_precond(mid, diag0, diag1, offdiag, x0, x1):
    """ApplyBroxPreconditioner.cpp:46-62 in FP32."""
    mid, diag0, diag1, offdiag, x0, x1 = (_c32(a) for a in (mid, diag0, diag1, offdiag, x0, x1))
    H, W = x0.shape
    y0, y1 = np.empty_like(x0), np.empty_like(x0)
    lib().hso_apply_brox_precond_f32(mid, diag0, diag1, offdiag, x0, x1, H, W, y0, y1)
    return y0, y1


BROX_OFFX = np.array([0, -1, 0, 1, 0], np.int32)   # top, left, mid, right, bottom
BROX_OFFY = np.array([-1, 0, 0, 0, 1], np.int32)


def hs_normal_matrix(lam, Ix, Iy):
    import scipy.sparse as sp

    Ix = np.asarray(Ix, np.float64)
    Iy = np.asarray(Iy, np.float64)
    H, W = Ix.shape

    def lap1(n):
        if n == 1:
            return sp.csr_matrix((1, 1))
        main = np.full(n, 2.0)
        main[0] = main[-1] = 1.0
        return sp.diags([main, -np.ones(n - 1), -np.ones(n - 1)], [0, -1, 1])

    L = sp.kron(sp.identity(H), lap1(W)) + sp.kron(lap1(H), sp.identity(W))
    ix, iy = Ix.ravel(), Iy.ravel()
    return sp.bmat([[sp.diags(ix * ix) + lam * L, sp.diags(ix * iy)],
                    [sp.diags(ix * iy), sp.diags(iy * iy) + lam * L]]).tocsr()


# ---------------------------------------------------------------- adjoint (FP64)

def hs_adjoint_f64(I0, I1, alpha, iters, lam_u, lam_v):
    """Reverse-mode gradient of L = <lam_u, u_K> + <lam_v, v_K> with respect to I0, I1
    and alpha, in FP64, storing every forward state (small sizes only).

    Forward sweep: ubar = A u; vbar = A v; r = Ix ubar + Iy vbar + It; d = a2 + Ix^2 + Iy^2;
    t = r / d; u' = ubar - Ix t; v' = vbar - Iy t.  Adjoint of one sweep, given the
    gradient (lu, lv) of its output: g = Ix lu + Iy lv; lr = -g/d; ld = g t / d;
    dIx += -lu t + lr ubar + 2 Ix ld; dIy += -lv t + lr vbar + 2 Iy ld; dIt += lr;
    da2 += ld; (lu, lv) <- A^T (lu + lr Ix, lv + lr Iy).  Then the derivative stencils'
    transposes map (dIx, dIy, dIt) to (dI0, dI1), and dalpha = 2 alpha da2.
    """
    f64 = np.float64
    I0 = np.asarray(I0, f64)
    I1 = np.asarray(I1, f64)
    Ix, Iy, It = hs_derivs(I0, I1, f64)
    a2 = f64(alpha) * f64(alpha)
    d = a2 + Ix * Ix + Iy * Iy
    avg = (AVG_W.astype(f64), AVG_OFFX, AVG_OFFY)
    u = np.zeros_like(I0)
    v = np.zeros_like(I0)
    states = []
    for _ in range(iters):
        states.append((u, v))
        ub = stencil2d(*avg, u, f64)
        vb = stencil2d(*avg, v, f64)
        t = (Ix * ub + Iy * vb + It) / d
        u, v = ub - Ix * t, vb - Iy * t
    lu = np.asarray(lam_u, f64).copy()
    lv = np.asarray(lam_v, f64).copy()
    dIx = np.zeros_like(I0)
    dIy = np.zeros_like(I0)
    dIt = np.zeros_like(I0)
    da2 = 0.0
    for k in range(iters - 1, -1, -1):
        uk, vk = states[k]
        ub = stencil2d(*avg, uk, f64)
        vb = stencil2d(*avg, vk, f64)
        t = (Ix * ub + Iy * vb + It) / d
        g = Ix * lu + Iy * lv
        lr = -g / d
        ldd = g * t / d
        dIx += -lu * t + lr * ub + 2 * Ix * ldd
        dIy += -lv * t + lr * vb + 2 * Iy * ldd
        dIt += lr
        da2 += ldd.sum()
        lu = stencil2d_transpose(*avg, lu + lr * Ix, f64)
        lv = stencil2d_transpose(*avg, lv + lr * Iy, f64)
    dxT = lambda w, z: stencil2d_transpose(w.astype(f64), D_OFFX, D_OFFY, z, f64)  # noqa: E731
    dI0 = dxT(DX_W, dIx) + dxT(DY_W, dIy) - dxT(DT_W, dIt)
    dI1 = dxT(DX_W, dIx) + dxT(DY_W, dIy) + dxT(DT_W, dIt)
    return dI0, dI1, 2.0 * f64(alpha) * da2, (u, v)



# ---------------------------------------------------------------- pyramid pieces (FP64)

BINOMIAL5 = np.array([1.0, 4.0, 6.0, 4.0, 1.0]) / 16.0


def blur_down(x):
    """5x5 binomial blur (separable [1 4 6 4 1]/16, clamp-to-edge taps), then keep every
    second pixel: out[y, x] = blur(x)[2y, 2x], shape (ceil(H/2), ceil(W/2))."""
    x = np.asarray(x, np.float64)
    H, W = x.shape
    Ho, Wo = (H + 1) // 2, (W + 1) // 2
    out = np.zeros((Ho, Wo))
    for dy in range(-2, 3):
        rr = np.clip(2 * np.arange(Ho) + dy, 0, H - 1)
        for dx in range(-2, 3):
            cc = np.clip(2 * np.arange(Wo) + dx, 0, W - 1)
            out += BINOMIAL5[dy + 2] * BINOMIAL5[dx + 2] * x[rr][:, cc]
    return out


def blur_down_adjoint(g, H, W):
    g = np.asarray(g, np.float64)
    Ho, Wo = g.shape
    out = np.zeros((H, W))
    for dy in range(-2, 3):
        rr = np.clip(2 * np.arange(Ho) + dy, 0, H - 1)
        for dx in range(-2, 3):
            cc = np.clip(2 * np.arange(Wo) + dx, 0, W - 1)
            np.add.at(out, (rr[:, None], cc[None, :]), BINOMIAL5[dy + 2] * BINOMIAL5[dx + 2] * g)
    return out


def _up_axis(n_fine, n_coarse):
    """Per fine index: (i0, i1, f) of the 2x bilinear upsampling with half-pixel centres
    (source coordinate (i + 0.5)/2 - 0.5), indices clamped into the coarse axis."""
    c = (np.arange(n_fine) + 0.5) / 2.0 - 0.5
    i0 = np.floor(c).astype(np.int64)
    f = c - i0
    return np.clip(i0, 0, n_coarse - 1), np.clip(i0 + 1, 0, n_coarse - 1), f


def upsample2(c, H, W, scale=2.0):
    """(H, W) = scale * bilinear 2x upsampling of c (Hc, Wc) with Hc = ceil(H/2)."""
    c = np.asarray(c, np.float64)
    Hc, Wc = c.shape
    y0, y1, fy = _up_axis(H, Hc)
    x0, x1, fx = _up_axis(W, Wc)
    fy, fx = fy[:, None], fx[None, :]
    return scale * ((1 - fy) * ((1 - fx) * c[y0][:, x0] + fx * c[y0][:, x1])
                    + fy * ((1 - fx) * c[y1][:, x0] + fx * c[y1][:, x1]))


def upsample2_adjoint(g, Hc, Wc, scale=2.0):
    g = np.asarray(g, np.float64)
    H, W = g.shape
    y0, y1, fy = _up_axis(H, Hc)
    x0, x1, fx = _up_axis(W, Wc)
    out = np.zeros((Hc, Wc))
    for yi, wy in ((y0, 1 - fy), (y1, fy)):
        for xi, wx in ((x0, 1 - fx), (x1, fx)):
            np.add.at(out, (yi[:, None], xi[None, :]), scale * wy[:, None] * wx[None, :] * g)
    return out


def warp_f64(src, ox, oy):
    """WarpImg2D.cpp:33-75 in exact FP64 arithmetic (no float roundings)."""
    src = np.asarray(src, np.float64)
    ox = np.asarray(ox, np.float64)
    oy = np.asarray(oy, np.float64)
    H, W = src.shape
    mx = np.floor(ox).astype(np.int64)
    my = np.floor(oy).astype(np.int64)
    xf, yf = ox - mx, oy - my
    Y, X = np.mgrid[0:H, 0:W]
    ok = (X + mx >= 0) & (X + mx + 1 < W) & (Y + my >= 0) & (Y + my + 1 < H)
    bx = np.where(ok, X + mx, 0)
    by = np.where(ok, Y + my, 0)
    bx1 = np.minimum(bx + 1, W - 1)
    by1 = np.minimum(by + 1, H - 1)
    o = (src[by, bx] * (1 - xf) * (1 - yf) + src[by, bx1] * xf * (1 - yf)
         + src[by1, bx] * (1 - xf) * yf + src[by1, bx1] * xf * yf)
    return np.where(ok, o, src)


def warp_adjoint_f64(src, ox, oy, g):
    """(dsrc, dox, doy) of <g, warp(src, ox, oy)> (piecewise derivative; the integer part
    and the in-bounds test are locally constant)."""
    src = np.asarray(src, np.float64)
    ox = np.asarray(ox, np.float64)
    oy = np.asarray(oy, np.float64)
    g = np.asarray(g, np.float64)
    H, W = src.shape
    mx = np.floor(ox).astype(np.int64)
    my = np.floor(oy).astype(np.int64)
    xf, yf = ox - mx, oy - my
    Y, X = np.mgrid[0:H, 0:W]
    ok = (X + mx >= 0) & (X + mx + 1 < W) & (Y + my >= 0) & (Y + my + 1 < H)
    bx = np.where(ok, X + mx, 0)
    by = np.where(ok, Y + my, 0)
    bx1 = np.minimum(bx + 1, W - 1)
    by1 = np.minimum(by + 1, H - 1)
    dsrc = np.zeros((H, W))
    go = np.where(ok, g, 0.0)
    for yy, xx, w in ((by, bx, (1 - xf) * (1 - yf)), (by, bx1, xf * (1 - yf)),
                      (by1, bx, (1 - xf) * yf), (by1, bx1, xf * yf)):
        np.add.at(dsrc, (yy, xx), w * go)
    dsrc += np.where(ok, 0.0, g)
    s00, s10, s01, s11 = src[by, bx], src[by, bx1], src[by1, bx], src[by1, bx1]
    dox = go * ((1 - yf) * (s10 - s00) + yf * (s11 - s01))
    doy = go * ((1 - xf) * (s01 - s00) + xf * (s11 - s10))
    return dsrc, dox, doy


def coarse_to_fine_f64(I0, I1, alpha, levels, iters):
    """FP64 coarse-to-fine Horn-Schunck composed of the pieces above (the composition of
    hindemith_b200.pyramid.coarse_to_fine): binomial pyramids, then from the coarsest
    level up: upsample the flow (x2), warp I1 by it, run `iters` sweeps from zero on the
    warped pair and add the increment.  HS sweeps are the C restatement in double."""
    p0 = [np.asarray(I0, np.float64)]
    p1 = [np.asarray(I1, np.float64)]
    for _ in range(levels - 1):
        p0.append(blur_down(p0[-1]))
        p1.append(blur_down(p1[-1]))
    u = v = None
    for lev in range(levels - 1, -1, -1):
        if u is None:
            u, v = c_hs_forward(p0[lev], p1[lev], alpha, iters, np.float64)
        else:
            H, W = p0[lev].shape
            uu, vv = upsample2(u, H, W), upsample2(v, H, W)
            du, dv = c_hs_forward(p0[lev], warp_f64(p1[lev], uu, vv), alpha, iters, np.float64)
            u, v = uu + du, vv + dv
    return u, v
