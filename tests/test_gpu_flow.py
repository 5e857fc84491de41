"""Lucas-Kanade and the Brox building blocks on the GPU against the FP32 restatement of the
reference templates (bit-exact) and the reference's golden vectors, directly and through
the @hm surface."""
import numpy as np
import pytest
import torch

from conftest import assert_bitexact, golden
from hindemith_b200 import SpMat2D, brox_offsets, hm
from hindemith_b200 import flow as FL
from hindemith_b200 import hindemith as HM
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu


def cuda32(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("shape,rad", [((1, 1), 1), ((9, 9), 2), ((40, 70), 5), ((131, 97), 3),
                                       ((64, 64), 16), ((200, 150), 1), ((77, 45), 4),
                                       ((33, 129), 7), ((300, 517), 5), ((96, 100), 16)])
def test_lk_bitexact(cuda, shape, rad):
    H, W = shape
    rng = np.random.default_rng(H + W + rad)
    err, Ix, Iy = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(3))
    du, dv = FL.lk_least_squares(cuda32(err), cuda32(Ix), cuda32(Iy), rad)
    rdu, rdv = O.c_lk_least_squares(err, Ix, Iy, rad)
    assert_bitexact(du.cpu().numpy(), rdu)
    assert_bitexact(dv.cpu().numpy(), rdv)


def test_lk_against_reference_template_golden(cuda):
    """hs_lk_least_squares against the reference's LKLeastSquares device template run as C
    (tests/golden/make_template_golden.py): bit-identical."""
    g = golden("tmpl_lk.npz")
    for i in range(int(g["n"])):
        du, dv = FL.lk_least_squares(cuda32(g[f"err_{i}"]), cuda32(g[f"Ix_{i}"]), cuda32(g[f"Iy_{i}"]),
                                     int(g[f"rad_{i}"]))
        torch.cuda.synchronize()
        assert_bitexact(du.cpu().numpy(), g[f"du_{i}"], f"case {i}")
        assert_bitexact(dv.cpu().numpy(), g[f"dv_{i}"], f"case {i}")


def test_brox_against_reference_golden(cuda):
    g = golden("brox.npz")
    offx, offy = brox_offsets()
    for i in range(int(g["n"])):
        H, W = g[f"psi_{i}"].shape
        A = FL.DeviceSpMat2D.from_host(SpMat2D(np.zeros((5, H, W), np.float32), offx, offy))
        FL.set_brox_matrix(A, cuda32(g[f"psi_{i}"]), float(g["alpha"]))
        ax = FL.spmv_dia2d(A, cuda32(g[f"x_{i}"]))
        y0, y1 = FL.apply_brox_preconditioner(A, *(cuda32(g[f"{k}_{i}"]) for k in ("d0", "d1", "od", "x0", "x1")))
        torch.cuda.synchronize()
        assert_bitexact(ax.cpu().numpy(), g[f"ax_{i}"])
        assert_bitexact(y0.cpu().numpy(), g[f"y0_{i}"])
        assert_bitexact(y1.cpu().numpy(), g[f"y1_{i}"])


def test_brox_against_reference_template_golden(cuda):
    """SetBroxMatrix, SetBroxRedblackMatrix, SpmvDIA2D and ApplyBroxPreconditioner against
    their device templates run as C: bit-identical (matrices start from random values)."""
    g = golden("tmpl_brox.npz")
    offx, offy = brox_offsets()
    for i in range(int(g["n"])):
        A = FL.DeviceSpMat2D.from_host(SpMat2D(g[f"A0_{i}"], offx, offy))
        FL.set_brox_matrix(A, cuda32(g[f"psi_{i}"]), float(g["alpha"]))
        ax = FL.spmv_dia2d(A, cuda32(g[f"x_{i}"]))
        y0, y1 = FL.apply_brox_preconditioner(A, *(cuda32(g[f"{k}_{i}"]) for k in ("d0", "d1", "od", "x0", "x1")))
        torch.cuda.synchronize()
        assert_bitexact(A.data().cpu().numpy(), g[f"A_{i}"], f"A {i}")
        assert_bitexact(ax.cpu().numpy(), g[f"ax_{i}"], f"ax {i}")
        assert_bitexact(y0.cpu().numpy(), g[f"y0_{i}"], f"y0 {i}")
        assert_bitexact(y1.cpu().numpy(), g[f"y1_{i}"], f"y1 {i}")
        ox4, oy4 = np.delete(offx, 2), np.delete(offy, 2)
        B = FL.DeviceSpMat2D.from_host(SpMat2D(g[f"R0_{i}"], ox4, oy4))
        adiag = FL.set_brox_redblack_matrix(B, cuda32(g[f"psi_{i}"]), float(g["alpha"]))
        torch.cuda.synchronize()
        assert_bitexact(B.data().cpu().numpy(), g[f"R_{i}"], f"R {i}")
        assert_bitexact(adiag.cpu().numpy(), g[f"adiag_{i}"], f"adiag {i}")


@pytest.mark.parametrize("shape", [(1, 1), (2, 7), (33, 65)])
def test_brox_matrix_and_spmv_bitexact(cuda, shape):
    H, W = shape
    rng = np.random.default_rng(H * W)
    psi = rng.uniform(0.1, 1, (H, W)).astype(np.float32)
    x = rng.standard_normal((H, W)).astype(np.float32)
    init = rng.standard_normal((5, H, W)).astype(np.float32)  # entries no pixel writes persist
    offx, offy = brox_offsets()
    A = FL.DeviceSpMat2D.from_host(SpMat2D(init, offx, offy))
    FL.set_brox_matrix(A, cuda32(psi), 0.3)
    ref = O.c_set_brox_matrix(psi, 0.3, init)
    assert_bitexact(A.data().cpu().numpy(), ref)
    assert_bitexact(FL.spmv_dia2d(A, cuda32(x)).cpu().numpy(), O.c_spmv_dia2d(ref, offx, offy, x))
    # the red-black form: 4 off-diagonals and the middle term apart
    ox4, oy4 = np.delete(offx, 2), np.delete(offy, 2)
    init4 = init[[0, 1, 3, 4]].copy()
    B = FL.DeviceSpMat2D.from_host(SpMat2D(init4, ox4, oy4))
    adiag = FL.set_brox_redblack_matrix(B, cuda32(psi), 0.3)
    ref4, rad = O.c_set_brox_matrix(psi, 0.3, init4, redblack=True)
    assert_bitexact(B.data().cpu().numpy(), ref4)
    assert_bitexact(adiag.cpu().numpy(), rad)


def lk_program(err, Ix, Iy):
    du, dv = lk_least_squares(err, Ix, Iy)  # noqa: F821 (the @hm surface's call)
    return du, dv


def brox_step(A, psi, alpha, x, d0, d1, od):
    set_brox_matrix(A, psi, alpha)  # noqa: F821
    ax = A * x
    r = x - ax
    y0, y1 = applyBroxPreconditioner(A, d0, d1, od, red(r), black(r))  # noqa: F821
    return y0 + y1, ax


@pytest.fixture
def defines():
    old = dict(HM.defines)
    yield HM.defines
    HM.defines.clear()
    HM.defines.update(old)


def test_hm_lk_program(cuda, defines):
    defines["RADIUS"] = 4
    rng = np.random.default_rng(2)
    err, Ix, Iy = (rng.standard_normal((50, 60)).astype(np.float32) for _ in range(3))
    du, dv = hm(lk_program)(err=err, Ix=Ix, Iy=Iy)
    rdu, rdv = O.c_lk_least_squares(err, Ix, Iy, 4)
    assert_bitexact(du, rdu)
    assert_bitexact(dv, rdv)


def test_hm_brox_step(cuda):
    rng = np.random.default_rng(3)
    H, W = 30, 41
    psi = rng.uniform(0.1, 1, (H, W)).astype(np.float32)
    x, d0, d1 = (rng.uniform(0.2, 1, (H, W)).astype(np.float32) for _ in range(3))
    od = rng.uniform(-0.05, 0.05, (H, W)).astype(np.float32)
    offx, offy = brox_offsets()
    A = SpMat2D(np.zeros((5, H, W), np.float32), offx, offy)
    alpha = np.float32(0.6)
    y, ax = hm(brox_step)(A=A, psi=psi, alpha=alpha, x=x, d0=d0, d1=d1, od=od)
    data = O.c_set_brox_matrix(psi, alpha, np.zeros((5, H, W), np.float32))
    rax = O.c_spmv_dia2d(data, offx, offy, x)
    r = x - rax
    Yi, Xi = np.indices((H, W))
    red_r = np.where((Xi + Yi) & 1, np.float32(0), r).astype(np.float32)
    black_r = np.where((Xi + Yi) & 1, r, np.float32(0)).astype(np.float32)
    y0, y1 = O.c_apply_brox_precond(data[2], d0, d1, od, red_r, black_r)
    assert_bitexact(ax, rax)
    assert_bitexact(y, y0 + y1)
