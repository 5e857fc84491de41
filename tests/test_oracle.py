"""The oracle is pinned before it is trusted: NumPy and C restatements against the
golden fixtures produced by the reference's own hlib.py (tests/golden/make_golden.py),
bit for bit, plus properties of the FP64 path."""
import numpy as np
import pytest

from conftest import assert_bitexact, golden, golden_files
from oracle import hs_oracle as O


@pytest.mark.parametrize("path", golden_files("stencil_*.npz"))
def test_stencil_golden(path):
    d = np.load(path)
    for i, (H, W) in enumerate(d["shapes"]):
        x, ref = d[f"x{i}"], d[f"out{i}"]
        assert_bitexact(O.stencil2d(d["weights"], d["offx"], d["offy"], x), ref, f"numpy {path} {i}")
        assert_bitexact(O.c_stencil2d(d["weights"], d["offx"], d["offy"], x), ref, f"C {path} {i}")


@pytest.mark.parametrize("path", golden_files("hs_*.npz"))
def test_hs_program_golden(path):
    d = np.load(path)
    Ix, Iy, It = O.hs_derivs(d["I0"], d["I1"])
    for a, name in ((Ix, "Ix"), (Iy, "Iy"), (It, "It")):
        assert_bitexact(a, d[name], name)
    cIx, cIy, cIt = O.c_hs_derivs(d["I0"], d["I1"])
    for a, name in ((cIx, "Ix"), (cIy, "Iy"), (cIt, "It")):
        assert_bitexact(a, d[name], "C " + name)
    z = np.zeros_like(d["I0"])
    n = int(d["sweeps"])
    u, v = O.hs_sweeps(Ix, Iy, It, d["alpha2"], n, z, z)
    assert_bitexact(u, d["u"], "u")
    assert_bitexact(v, d["v"], "v")
    cu, cv = O.c_hs_sweeps(Ix, Iy, It, float(d["alpha2"]), n, z, z)
    assert_bitexact(cu, d["u"], "C u")
    assert_bitexact(cv, d["v"], "C v")


def test_warp_golden():
    """hlib.warp_img2d agrees with WarpImg2D.cpp for integer offsets except on the last
    row/column when that axis's offset is 0: the device template demands x+dx+1 < W
    (it always reads the 2x2 footprint) and keeps the source pixel there, while
    warp_img2d steps by sign(0) = 0.  The oracle follows the device template."""
    for name in ("warp_int.npz", "warp_zero.npz"):
        d = golden(name)
        src, ox, oy, ref = d["src"], d["ox"], d["oy"], d["out"]
        H, W = src.shape
        Y, X = np.mgrid[0:H, 0:W]
        device_rule = ((ox == 0) & (oy != 0) & (X == W - 1)) | ((oy == 0) & (ox != 0) & (Y == H - 1))
        for fn in (O.warp, O.c_warp):
            out = fn(src, ox, oy)
            np.testing.assert_array_equal(out[~device_rule], ref[~device_rule])
            np.testing.assert_array_equal(out[device_rule], src[device_rule])


def test_warp_matches_reference_template_golden():
    """Fractional offsets (integer, -0 and tiny negative ones among them) against the
    reference's WarpImg2D device template run as C (tests/golden/make_template_golden.py):
    both restatements bit-identical, C's left-to-right float/double typing included."""
    g = golden("tmpl_warp.npz")
    for i in range(int(g["n"])):
        src, ox, oy = g[f"src_{i}"], g[f"ox_{i}"], g[f"oy_{i}"]
        assert_bitexact(O.c_warp(src, ox, oy), g[f"out_{i}"], f"C, case {i}")
        assert_bitexact(O.warp(src, ox, oy), g[f"out_{i}"], f"NumPy, case {i}")


def test_matrix_powers_matches_reference_template_golden():
    """HSMatrixPowers' device template (copy into plane 0, one launch per step) run as C
    (tests/golden/make_template_golden.py) against the C restatement: bit-identical."""
    g = golden("tmpl_matrix_powers.npz")
    for i in range(int(g["n"])):
        V0, V1 = O.c_hs_matrix_powers(g[f"lam_{i}"], g[f"Ix_{i}"], g[f"Iy_{i}"], g[f"r0_{i}"],
                                      g[f"r1_{i}"], int(g[f"steps_{i}"]))
        assert_bitexact(V0, g[f"V0_{i}"], f"V0, case {i}")
        assert_bitexact(V1, g[f"V1_{i}"], f"V1, case {i}")


def test_warp_fractional_numpy_vs_c():
    rng = np.random.default_rng(3)
    src = rng.random((23, 29), dtype=np.float32)
    ox = (rng.random((23, 29)) * 8 - 4).astype(np.float32)
    oy = (rng.random((23, 29)) * 8 - 4).astype(np.float32)
    assert_bitexact(O.warp(src, ox, oy), O.c_warp(src, ox, oy), "warp")


def test_fp64_oracle_close_to_fp32():
    from hindemith_b200 import synthetic

    I0, I1, _, _ = synthetic.make_pair(64, 80, seed=1000)
    u32, v32 = O.c_hs_forward(I0, I1, 1.0, 100, np.float32)
    u64, v64 = O.c_hs_forward(I0, I1, 1.0, 100, np.float64)
    assert np.abs(u32 - u64).max() < 1e-5
    assert np.abs(v32 - v64).max() < 1e-5
    un, vn = O.hs_forward(I0, I1, 1.0, 100, np.float64)
    np.testing.assert_allclose(un, u64, rtol=0, atol=1e-12)


def test_numpy_and_c_forward_agree_bitwise():
    from hindemith_b200 import synthetic

    I0, I1, _, _ = synthetic.make_pair(37, 53, seed=1001)
    a = O.hs_forward(I0, I1, 0.7, 25, np.float32)
    b = O.c_hs_forward(I0, I1, 0.7, 25, np.float32)
    assert_bitexact(a[0], b[0], "u")
    assert_bitexact(a[1], b[1], "v")


def test_known_answers():
    # a constant image has zero derivatives, so the flow stays exactly 0
    c = np.full((9, 11), 0.37, dtype=np.float32)
    u, v = O.c_hs_forward(c, c, 1.0, 50)
    assert not u.any() and not v.any()
    # a horizontal ramp translated by s: It/Ix = -s in the interior, and with a small
    # alpha the interior flow approaches (s, 0)
    H, W, s = 24, 40, 0.5
    x = np.arange(W, dtype=np.float64)
    I0 = np.tile(0.02 * x, (H, 1)).astype(np.float32)
    I1 = np.tile(0.02 * (x - s), (H, 1)).astype(np.float32)
    Ix, Iy, It = O.c_hs_derivs(I0, I1, np.float64)
    mid = (slice(2, -2), slice(2, -2))
    np.testing.assert_allclose(It[mid] / Ix[mid], -s, atol=1e-6)
    u, v = O.c_hs_forward(I0, I1, 0.01, 2000, np.float64)
    assert np.abs(u[8:-8, 8:-8] - s).max() < 1e-3
    assert np.abs(v).max() < 1e-6


def test_stencil_transpose_adjoint():
    """<S x, y> = <x, S^T y> in FP64 for clamp-to-edge stencils."""
    rng = np.random.default_rng(5)
    for (H, W) in ((1, 1), (1, 6), (5, 1), (7, 9)):
        x = rng.standard_normal((H, W))
        y = rng.standard_normal((H, W))
        for w, ox, oy in ((O.AVG_W, O.AVG_OFFX, O.AVG_OFFY), (O.DX_W, O.D_OFFX, O.D_OFFY)):
            w = w.astype(np.float64)
            Sx = O.c_stencil2d(w, ox, oy, x, np.float64)
            STy = O.c_stencil2d_transpose(w, ox, oy, y)
            assert abs((Sx * y).sum() - (x * STy).sum()) < 1e-12
            np.testing.assert_allclose(STy, O.stencil2d_transpose(w, ox, oy, y), atol=1e-14)


def test_torch_reference_matches_fp64_oracle():
    """The pure-PyTorch HS used as a gradient reference agrees with the FP64 oracle in
    both the forward and the reverse mode."""
    import torch

    from hs_torch_ref import hs_torch

    rng = np.random.default_rng(11)
    H, W, K = 13, 17, 15
    from hindemith_b200 import synthetic

    I0, I1, _, _ = synthetic.make_pair(H, W, seed=4)
    lu, lv = rng.standard_normal((H, W)), rng.standard_normal((H, W))
    t0 = torch.from_numpy(I0.astype(np.float64)).requires_grad_(True)
    t1 = torch.from_numpy(I1.astype(np.float64)).requires_grad_(True)
    ta = torch.tensor(0.6, dtype=torch.float64, requires_grad=True)
    u, v = hs_torch(t0, t1, ta, K)
    ((u * torch.from_numpy(lu)).sum() + (v * torch.from_numpy(lv)).sum()).backward()
    r0, r1, ra, (ru, rv) = O.hs_adjoint_f64(I0, I1, 0.6, K, lu, lv)
    np.testing.assert_allclose(u.detach().numpy(), ru, atol=1e-12)
    np.testing.assert_allclose(t0.grad.numpy(), r0, atol=1e-10)
    np.testing.assert_allclose(t1.grad.numpy(), r1, atol=1e-10)
    assert abs(float(ta.grad) - ra) < 1e-9


def test_pyramid_adjoints_dot_product():
    """<A x, y> = <x, A^T y> for blur-down and 2x upsampling; FD for the warp offsets."""
    rng = np.random.default_rng(21)
    for H, W in ((1, 1), (2, 3), (5, 8), (9, 7), (16, 16)):
        x = rng.standard_normal((H, W))
        y = rng.standard_normal(((H + 1) // 2, (W + 1) // 2))
        assert abs((O.blur_down(x) * y).sum() - (x * O.blur_down_adjoint(y, H, W)).sum()) < 1e-12
        c = rng.standard_normal(((H + 1) // 2, (W + 1) // 2))
        z = rng.standard_normal((H, W))
        assert abs((O.upsample2(c, H, W) * z).sum()
                   - (c * O.upsample2_adjoint(z, c.shape[0], c.shape[1])).sum()) < 1e-12
    H, W = 12, 15
    src = rng.random((H, W))
    ox = rng.uniform(-3, 3, (H, W))
    oy = rng.uniform(-3, 3, (H, W))
    g = rng.standard_normal((H, W))
    dsrc, dox, doy = O.warp_adjoint_f64(src, ox, oy, g)
    s2 = rng.standard_normal((H, W))
    assert abs((O.warp_f64(s2, ox, oy) * g).sum() - (s2 * dsrc).sum()) < 1e-12
    h = 1e-6
    for i, j in ((3, 4), (6, 7), (10, 2)):
        for arr, d in ((ox, dox), (oy, doy)):
            p, m = arr.copy(), arr.copy()
            p[i, j] += h
            m[i, j] -= h
            fp = O.warp_f64(src, p, oy) if arr is ox else O.warp_f64(src, ox, p)
            fm = O.warp_f64(src, m, oy) if arr is ox else O.warp_f64(src, ox, m)
            fd = ((fp - fm) * g).sum() / (2 * h)
            assert abs(fd - d[i, j]) < 1e-6
    # the FP64 warp agrees with the FP32-rounding restatement to float precision
    assert np.abs(O.warp_f64(src, ox, oy) - O.warp(src, ox, oy)).max() < 1e-6


def test_torch_pyramid_reference_matches_oracle():
    import torch
    from hs_torch_ref import blur_down_torch, upsample2_torch, warp_torch

    rng = np.random.default_rng(17)
    for H, W in [(1, 1), (5, 4), (37, 53)]:
        x = rng.standard_normal((H, W))
        c = O.blur_down(x)
        assert np.array_equal(blur_down_torch(torch.tensor(x)).numpy(), c)
        np.testing.assert_allclose(upsample2_torch(torch.tensor(c), H, W).numpy(),
                                   O.upsample2(c, H, W), rtol=0, atol=1e-14)
        ox, oy = rng.uniform(-3, 3, (H, W)), rng.uniform(-3, 3, (H, W))
        np.testing.assert_allclose(warp_torch(torch.tensor(x), torch.tensor(ox), torch.tensor(oy)).numpy(),
                                   O.warp_f64(x, ox, oy), rtol=0, atol=1e-14)


def test_hs_average_is_self_adjoint():
    """A^T = A for the clamp-to-edge 3x3 HS average (what lets the adjoint sweep stream
    with the forward's skeleton): the transposed stencil equals the stencil itself."""
    rng = np.random.default_rng(11)
    w = O.AVG_W.astype(np.float64)
    for (H, W) in ((1, 1), (1, 5), (4, 1), (2, 2), (3, 7), (16, 13)):
        y = rng.standard_normal((H, W))
        np.testing.assert_allclose(O.c_stencil2d_transpose(w, O.AVG_OFFX, O.AVG_OFFY, y),
                                   O.c_stencil2d(w, O.AVG_OFFX, O.AVG_OFFY, y, np.float64),
                                   rtol=0, atol=1e-15)


def test_stencil_precond_brox_oracles_match_reference_templates():
    """Stencil2DMVM, ApplyHSPreconditioner (determinants at float(1e-15)), SetBroxMatrix,
    SetBroxRedblackMatrix, SpmvDIA2D and ApplyBroxPreconditioner: the reference's device
    templates run as C (tests/golden/make_template_golden.py) against the restatements."""
    g = golden("tmpl_stencil.npz")
    for i in range(int(g["n"])):
        args = (g[f"w_{i}"], g[f"offx_{i}"], g[f"offy_{i}"], g[f"x_{i}"])
        assert_bitexact(O.c_stencil2d(*args), g[f"out_{i}"], f"stencil C {i}")
        assert_bitexact(O.stencil2d(*args), g[f"out_{i}"], f"stencil NumPy {i}")
    g = golden("tmpl_precond.npz")
    for i in range(int(g["n"])):
        y0, y1 = O.c_apply_hs_precond(g[f"s2_{i}"], *(g[f"{k}_{i}"] for k in ("d0", "d1", "od", "x0", "x1")))
        assert_bitexact(y0, g[f"y0_{i}"], f"precond {i}")
        assert_bitexact(y1, g[f"y1_{i}"], f"precond {i}")
    g = golden("tmpl_brox.npz")
    for i in range(int(g["n"])):
        assert_bitexact(O.c_set_brox_matrix(g[f"psi_{i}"], g["alpha"], g[f"A0_{i}"]), g[f"A_{i}"])
        R, adiag = O.c_set_brox_matrix(g[f"psi_{i}"], g["alpha"], g[f"R0_{i}"], redblack=True)
        assert_bitexact(R, g[f"R_{i}"])
        assert_bitexact(adiag, g[f"adiag_{i}"])
        assert_bitexact(O.c_spmv_dia2d(g[f"A_{i}"], O.BROX_OFFX, O.BROX_OFFY, g[f"x_{i}"]), g[f"ax_{i}"])
        y0, y1 = O.c_apply_brox_precond(g[f"A_{i}"][2], *(g[f"{k}_{i}"] for k in ("d0", "d1", "od", "x0", "x1")))
        assert_bitexact(y0, g[f"y0_{i}"])
        assert_bitexact(y1, g[f"y1_{i}"])


def test_precond_oracle_matches_reference_golden():
    """ApplyHSPreconditioner restatement vs hlib.applyHSPreconditioner (golden fixtures):
    bit-identical where both determinant guards agree (all of the fixtures)."""
    for name in ("precond_rand", "precond_zero"):
        g = golden(name + ".npz")
        for i in range(int(g["n"])):
            y0, y1 = O.c_apply_hs_precond(g["s2"], g[f"d0_{i}"], g[f"d1_{i}"], g[f"od_{i}"],
                                          g[f"x0_{i}"], g[f"x1_{i}"])
            assert_bitexact(y0, g[f"y0_{i}"])
            assert_bitexact(y1, g[f"y1_{i}"])


def test_matrix_powers_oracle_matches_sparse_operator():
    """HSMatrixPowers restatement vs the HS normal-equations operator assembled
    independently as a sparse FP64 matrix (FP32 vs FP64: 1e-5 relative)."""
    rng = np.random.default_rng(23)
    for (H, W) in ((1, 1), (1, 6), (5, 1), (9, 13)):
        Ix, Iy, r0, r1 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(4))
        lam = np.float32(0.8)
        V0, V1 = O.c_hs_matrix_powers(lam, Ix, Iy, r0, r1, 5)
        M = O.hs_normal_matrix(np.float64(lam), Ix, Iy)
        x = np.concatenate([r0.ravel(), r1.ravel()]).astype(np.float64)
        for s in range(5):
            ref = x / max(np.abs(x).max(), 1e-30)
            got = np.concatenate([V0[s].ravel(), V1[s].ravel()]) / max(np.abs(x).max(), 1e-30)
            assert np.abs(got - ref).max() < 1e-5
            x = M @ x


def test_brox_oracle_matches_reference_golden():
    """set_brox_matrix + SpMat2D product and applyBroxPreconditioner (hlib.py:49-81,
    148-164) vs the restatement of the device templates: bit-identical.  (hlib indexes each
    diagonal by the row of its entry, the device templates by its column; the product is
    the same either way.)"""
    g = golden("brox.npz")
    for i in range(int(g["n"])):
        H, W = g[f"psi_{i}"].shape
        data = O.c_set_brox_matrix(g[f"psi_{i}"], g["alpha"], np.zeros((5, H, W), np.float32))
        assert_bitexact(O.c_spmv_dia2d(data, O.BROX_OFFX, O.BROX_OFFY, g[f"x_{i}"]), g[f"ax_{i}"])
        assert_bitexact(data[2], g[f"mid_{i}"])
        y0, y1 = O.c_apply_brox_precond(data[2], g[f"d0_{i}"], g[f"d1_{i}"], g[f"od_{i}"],
                                        g[f"x0_{i}"], g[f"x1_{i}"])
        assert_bitexact(y0, g[f"y0_{i}"])
        assert_bitexact(y1, g[f"y1_{i}"])


def test_lk_oracle_matches_reference_template_golden():
    """The LKLeastSquares restatement against the reference's own device template
    (LKLeastSquares.cpp:39-91), instantiated as C by tests/golden/make_template_golden.py:
    bit-identical, including the border rule and det == 0 windows."""
    g = golden("tmpl_lk.npz")
    for i in range(int(g["n"])):
        du, dv = O.c_lk_least_squares(g[f"err_{i}"], g[f"Ix_{i}"], g[f"Iy_{i}"], int(g[f"rad_{i}"]))
        assert_bitexact(du, g[f"du_{i}"], f"case {i}")
        assert_bitexact(dv, g[f"dv_{i}"], f"case {i}")


def test_lk_oracle_matches_float64_restatement():
    """The LKLeastSquares restatement against an independent FP64 NumPy evaluation of the
    same template (window [-r, r)^2, interior rule).  (The reference's NumPy
    lk_least_squares, hlib.py:86-118, is a different algorithm with a (2r+1)^2 window.)"""
    rng = np.random.default_rng(9)
    for (H, W, r) in ((12, 15, 2), (20, 9, 3), (5, 5, 2)):
        err, Ix, Iy = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(3))
        du, dv = O.c_lk_least_squares(err, Ix, Iy, r)
        rdu, rdv = np.zeros((H, W)), np.zeros((H, W))
        for y in range(r, H - r):
            for x in range(r, W - r):
                a = Ix[y - r:y + r, x - r:x + r].astype(np.float64)
                b = Iy[y - r:y + r, x - r:x + r].astype(np.float64)
                e = err[y - r:y + r, x - r:x + r].astype(np.float64)
                M = np.array([[(a * a).sum(), (a * b).sum()], [(a * b).sum(), (b * b).sum()]])
                rhs = np.array([(a * e).sum(), (b * e).sum()])
                rdu[y, x], rdv[y, x] = np.linalg.solve(M, rhs)
        scale = max(np.abs(rdu).max(), np.abs(rdv).max(), 1e-6)
        assert np.abs(du - rdu).max() < 1e-4 * scale
        assert np.abs(dv - rdv).max() < 1e-4 * scale


def test_coarse_to_fine_f64_matches_torch_float64():
    """The FP64 coarse-to-fine composition the benchmark checks config-4 flows against
    equals the float64 PyTorch composition of the same pieces."""
    import torch

    from hindemith_b200 import synthetic
    from hs_torch_ref import coarse_to_fine_torch

    I0, I1, _, _ = synthetic.make_pair(48, 64, seed=21, amplitude=4.0)
    u, v = O.coarse_to_fine_f64(I0, I1, 1.0, 3, 15)
    ur, vr = coarse_to_fine_torch(torch.from_numpy(I0.astype(np.float64)),
                                  torch.from_numpy(I1.astype(np.float64)), 1.0, 3, 15)
    assert np.abs(u - ur.numpy()).max() < 1e-9 and np.abs(v - vr.numpy()).max() < 1e-9
