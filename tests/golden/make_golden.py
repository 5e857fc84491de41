"""Generate the golden fixtures from the reference's own CPU code (run in a container
that holds the reference checkout; the fixtures are committed, this script is not run
by the tests).

    python tests/golden/make_golden.py <path of the reference checkout>

The reference's only CPU implementation of the path is its NumPy library, hlib.py
(Stencil.__mul__ at hlib.py:173-191, warp_img2d at hlib.py:120-138).  It is Python 2
code; it is loaded here unchanged, from an in-memory copy, with three adjustments to
the *environment* it ran in (not to its code):
  * tabs are expanded to 8 columns (Python 2's rule; Python 3 rejects mixed indents);
  * `min` / `max` / `round` are rebound to the builtins: under NumPy 2,
    `from numpy import *` also exports NumPy's min/max/round, which NumPy 1.x (the
    reference's era) did not, and Stencil.__mul__ calls the builtins on tap lists;
  * `sign` returns an int: warp_img2d indexes with `v_int + i + sign(v)`, a float
    index that NumPy 1.x truncated and NumPy 2 rejects.

hlib.Stencil.__mul__ pads with max(|offset|) per side and so only works for symmetric
tap sets.  An asymmetric stencil such as the 2x2 derivative taps over {0,1}^2 is made
symmetric by prepending a zero-weight tap at (-1, -1): the padding then matches, the
first accumulation is 0 + 0*x = +0 exactly, and every later rounding is unchanged.

Fixtures (tests/golden/*.npz):
  stencil_*.npz  : x, weights, offx, offy, out      (Stencil * Array2D)
  hs_*.npz       : I0, I1, alpha2, sweeps, Ix, Iy, It, u, v   (hs_programs.hs_jacobi)
  warp_*.npz     : src, ox, oy, out                 (warp_img2d, integer offsets)
  precond_*.npz  : s2, d0_i, d1_i, od_i, x0_i, x1_i, y0_i, y1_i   (applyHSPreconditioner)
  brox.npz       : alpha, psi_i, x_i, ax_i (set_brox_matrix then A*x), mid_i, d0_i, d1_i,
                   od_i, x0_i, x1_i, y0_i, y1_i (applyBroxPreconditioner)
"""
from __future__ import annotations

import builtins
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import hs_programs  # noqa: E402


def load_reference_hlib(ref_root: str):
    path = os.path.join(ref_root, "hlib.py")
    src = open(path).read().expandtabs(8)
    mod = types.ModuleType("hlib_reference")
    exec(compile(src, path, "exec"), mod.__dict__)
    for name in ("min", "max", "round"):
        mod.__dict__[name] = getattr(builtins, name)
    mod.__dict__["sign"] = lambda a: int(np.sign(a))
    return mod


def symmetric(hl, w, ox, oy):
    """hlib Stencil for taps (w, ox, oy); a zero tap at (-1,-1) first if asymmetric."""
    w = np.asarray(w, dtype=np.float32)
    ox = np.asarray(ox, dtype=np.int64)
    oy = np.asarray(oy, dtype=np.int64)
    sym_x = -min(0, ox.min()) == max(0, ox.max())
    sym_y = -min(0, oy.min()) == max(0, oy.max())
    if not (sym_x and sym_y):
        w = np.concatenate([np.float32([0.0]), w])
        ox = np.concatenate([[-1], ox])
        oy = np.concatenate([[-1], oy])
    return hl.Stencil(w, ox, oy)


AVG = ([1 / 12, 1 / 6, 1 / 12, 1 / 6, 1 / 6, 1 / 12, 1 / 6, 1 / 12],
       [-1, 0, 1, -1, 1, -1, 0, 1], [-1, -1, -1, 0, 0, 1, 1, 1])
D_OX, D_OY = [0, 1, 0, 1], [0, 0, 1, 1]
DX = ([-0.25, 0.25, -0.25, 0.25], D_OX, D_OY)
DY = ([-0.25, -0.25, 0.25, 0.25], D_OX, D_OY)
DT = ([0.25, 0.25, 0.25, 0.25], D_OX, D_OY)


def binomial5():
    k = np.array([1, 4, 6, 4, 1], dtype=np.float64) / 16
    w, ox, oy = [], [], []
    for dy in range(-2, 3):
        for dx in range(-2, 3):
            w.append(k[dy + 2] * k[dx + 2])
            ox.append(dx)
            oy.append(dy)
    return w, ox, oy


def laplace9():
    w, ox, oy = [], [], []
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            w.append(-8.0 if (dx, dy) == (0, 0) else 1.0)
            ox.append(dx)
            oy.append(dy)
    return w, ox, oy


def main(ref_root: str):
    hl = load_reference_hlib(ref_root)
    rng = np.random.Generator(np.random.PCG64(7))
    out_dir = HERE

    stencils = {"avg": AVG, "dx": DX, "dt": DT, "binomial5": binomial5(), "laplace9": laplace9()}
    shapes = [(1, 1), (1, 7), (7, 1), (2, 2), (13, 17)]
    for sname, (w, ox, oy) in stencils.items():
        xs, outs = [], []
        for (H, W) in shapes:
            x = rng.random((H, W), dtype=np.float32) * np.float32(2) - np.float32(0.5)
            y = symmetric(hl, w, ox, oy) * x
            assert y.dtype == np.float32
            xs.append(x)
            outs.append(y)
        np.savez_compressed(os.path.join(out_dir, f"stencil_{sname}.npz"),
                            weights=np.asarray(w, dtype=np.float32),
                            offx=np.asarray(ox, dtype=np.int32), offy=np.asarray(oy, dtype=np.int32),
                            shapes=np.asarray(shapes, dtype=np.int32),
                            **{f"x{i}": a for i, a in enumerate(xs)},
                            **{f"out{i}": a for i, a in enumerate(outs)})

    # Horn-Schunck programs under the reference's NumPy semantics
    cases = [("1x1", 1, 1, 3), ("2x2", 2, 2, 5), ("1x9", 1, 9, 7), ("9x1", 9, 1, 7),
             ("24x31", 24, 31, 20), ("33x65", 33, 65, 100), ("70x130", 70, 130, 37)]
    Dx, Dy, Dt = (symmetric(hl, *s) for s in (DX, DY, DT))
    A = symmetric(hl, *AVG)
    from scipy.ndimage import gaussian_filter
    for name, H, W, sweeps in cases:
        I0 = gaussian_filter(rng.random((H, W)), 1.5, mode="reflect").astype(np.float32)
        I1 = (np.roll(I0, 1, axis=1) + rng.normal(0, 0.01, (H, W))).astype(np.float32)
        alpha2 = np.float32(rng.uniform(0.3, 2.0)) ** 2
        z = np.zeros((H, W), dtype=np.float32)
        u, v = hs_programs.hs_jacobi(I0=I0, I1=I1, Dx=Dx, Dy=Dy, Dt=Dt, A=A,
                                     alpha2=np.float32(alpha2), u=z, v=z, sweeps=sweeps)
        Ix = Dx * I0 + Dx * I1
        Iy = Dy * I0 + Dy * I1
        It = Dt * I1 - Dt * I0
        assert u.dtype == np.float32 and v.dtype == np.float32
        np.savez_compressed(os.path.join(out_dir, f"hs_{name}.npz"), I0=I0, I1=I1,
                            alpha2=np.float32(alpha2), sweeps=np.int32(sweeps), Ix=Ix, Iy=Iy,
                            It=It, u=u, v=v)

    # warp_img2d agrees with WarpImg2D.cpp for integer offsets; record those
    H, W = 16, 20
    src = rng.random((H, W), dtype=np.float32)
    flows = {"int": (rng.integers(-3, 4, (H, W)), rng.integers(-3, 4, (H, W))),
             "zero": (np.zeros((H, W), np.int64), np.zeros((H, W), np.int64))}
    for fname, (ox, oy) in flows.items():
        out = hl.warp_img2d(src, ox.astype(np.float64), oy.astype(np.float64))
        np.savez_compressed(os.path.join(out_dir, f"warp_{fname}.npz"), src=src,
                            ox=ox.astype(np.float32), oy=oy.astype(np.float32),
                            out=np.asarray(out, dtype=np.float32))
    # applyHSPreconditioner (hlib.py:18-47): the block-Jacobi step of the HS system.  Its
    # determinant guard (|det| > 1e-4) differs from the device template's (> 1e-15); the
    # random case keeps every |det| above 1e-4 so that both guards agree, and the zero
    # case has det = 0 exactly (both copy x through).
    prng = np.random.Generator(np.random.PCG64(11))
    for cname, scale in (("rand", 1.0), ("zero", 0.0)):
        arrs = {}
        for i, (H, W) in enumerate([(1, 1), (1, 5), (6, 1), (13, 17)]):
            d0 = (prng.uniform(0.1, 1.0, (H, W)) * scale).astype(np.float32)
            d1 = (prng.uniform(0.1, 1.0, (H, W)) * scale).astype(np.float32)
            od = (prng.uniform(-0.05, 0.05, (H, W)) * scale).astype(np.float32)
            x0 = prng.standard_normal((H, W)).astype(np.float32)
            x1 = prng.standard_normal((H, W)).astype(np.float32)
            sdata = np.float32([0.0, 0.0, 0.25 * scale, 0.0])
            D = hl.Stencil(sdata, np.int64([0, 1, 0, 1]), np.int64([0, 0, 1, 1]))
            y0, y1 = hl.applyHSPreconditioner(D, d0, d1, od, x0, x1)
            arrs.update({f"d0_{i}": d0, f"d1_{i}": d1, f"od_{i}": od, f"x0_{i}": x0,
                         f"x1_{i}": x1, f"y0_{i}": np.asarray(y0, np.float32),
                         f"y1_{i}": np.asarray(y1, np.float32)})
        np.savez_compressed(os.path.join(out_dir, f"precond_{cname}.npz"),
                            s2=np.float32(0.25 * scale), n=np.int32(4), **arrs)
    # Brox: set_brox_matrix (hlib.py:71-81) then the SpMat2D product (hlib.py:148-164),
    # and applyBroxPreconditioner (hlib.py:49-69).  hlib stores each diagonal at the row of
    # the matrix entry, the device templates at its column; A*x agrees between the two.
    brng = np.random.Generator(np.random.PCG64(13))
    arrs = {}
    shapes = [(1, 1), (1, 6), (5, 1), (9, 14)]
    offx = np.array([0, -1, 0, 1, 0])
    offy = np.array([-1, 0, 0, 0, 1])
    for i, (H, W) in enumerate(shapes):
        psi = brng.uniform(0.1, 1.0, (H, W)).astype(np.float32)
        x = brng.standard_normal((H, W)).astype(np.float32)
        Am = hl.SpMat2D(np.zeros((5, H, W), np.float32), offx, offy)
        alpha = np.float32(0.75)
        hl.set_brox_matrix(Am, psi, alpha)
        ax = Am * x
        d0 = brng.uniform(0.1, 1.0, (H, W)).astype(np.float32)
        d1 = brng.uniform(0.1, 1.0, (H, W)).astype(np.float32)
        od = brng.uniform(-0.05, 0.05, (H, W)).astype(np.float32)
        x0 = brng.standard_normal((H, W)).astype(np.float32)
        x1 = brng.standard_normal((H, W)).astype(np.float32)
        y0, y1 = hl.applyBroxPreconditioner(Am, d0, d1, od, x0, x1)
        arrs.update({f"psi_{i}": psi, f"x_{i}": x, f"ax_{i}": np.asarray(ax, np.float32),
                     f"mid_{i}": Am.data[2].copy(), f"d0_{i}": d0, f"d1_{i}": d1, f"od_{i}": od,
                     f"x0_{i}": x0, f"x1_{i}": x1, f"y0_{i}": np.asarray(y0, np.float32),
                     f"y1_{i}": np.asarray(y1, np.float32)})
    np.savez_compressed(os.path.join(out_dir, "brox.npz"), alpha=np.float32(0.75),
                        n=np.int32(len(shapes)), **arrs)
    print("wrote fixtures to", out_dir)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
