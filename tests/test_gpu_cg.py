"""Horn-Schunck as a linear system on the GPU: hs_matrix_powers and
hs_apply_hs_preconditioner against the FP32 restatement (bit-exact) and the reference's
golden vectors, and the preconditioned CG solver against a sparse FP64 direct solve."""
import numpy as np
import pytest
import torch

from conftest import assert_bitexact, golden
from hindemith_b200 import _lib as L
from hindemith_b200 import cg
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu


def cuda32(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("depth", [1, 3, 4])
def test_matrix_powers_against_reference_template_golden(cuda, depth):
    """hs_matrix_powers against the reference's HSMatrixPowers device template run as C
    (copy into plane 0, one launch per step): bit-identical at every pass depth."""
    g = golden("tmpl_matrix_powers.npz")
    for i in range(int(g["n"])):
        steps = int(g[f"steps_{i}"])
        V0, V1 = cg.hs_matrix_powers(float(g[f"lam_{i}"]), *(cuda32(g[f"{k}_{i}"]) for k in ("Ix", "Iy", "r0", "r1")),
                                     steps, L.make_config(sweeps_per_pass=depth))
        torch.cuda.synchronize()
        for s in range(steps):
            assert_bitexact(V0[s].cpu().numpy(), g[f"V0_{i}"][s], f"case {i} V0[{s}]")
            assert_bitexact(V1[s].cpu().numpy(), g[f"V1_{i}"][s], f"case {i} V1[{s}]")


@pytest.mark.parametrize("shape", [(1, 1), (1, 5), (6, 1), (2, 3), (33, 65), (100, 130), (257, 96),
                                   (150, 250), (300, 517)])  # the last two have interior tiles
@pytest.mark.parametrize("depth", [1, 2, 3, 4])
def test_matrix_powers_bitexact(cuda, shape, depth):
    H, W = shape
    rng = np.random.default_rng(H * 7 + W + depth)
    Ix, Iy, r0, r1 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(4))
    lam = np.float32(0.65)
    steps = 7
    V0, V1 = cg.hs_matrix_powers(float(lam), cuda32(Ix), cuda32(Iy), cuda32(r0), cuda32(r1), steps,
                                 L.make_config(sweeps_per_pass=depth))
    torch.cuda.synchronize()
    R0, R1 = O.c_hs_matrix_powers(lam, Ix, Iy, r0, r1, steps)
    for s in range(steps):
        assert_bitexact(V0[s].cpu().numpy(), R0[s], f"V0[{s}]")
        assert_bitexact(V1[s].cpu().numpy(), R1[s], f"V1[{s}]")


@pytest.mark.parametrize("depth", [3, 4])
def test_matrix_powers_large_and_in_place(cuda, depth):
    """Many strips and segments (1000x1500, ld padded), and V[0] given as r itself: the
    powers still equal the FP32 restatement bit for bit."""
    import ctypes

    from hindemith_b200 import device as D

    H, W, steps = 1000, 1498, 9
    rng = np.random.default_rng(depth)
    Ix, Iy, r0, r1 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(4))
    lam = np.float32(0.4)
    R0, R1 = O.c_hs_matrix_powers(lam, Ix, Iy, r0, r1, steps)
    Ixd, Iyd = D.as_plane(cuda32(Ix)), D.as_plane(cuda32(Iy))
    ld = D.ld_of(Ixd)
    buf = torch.empty((2, steps, H, ld), dtype=torch.float32, device="cuda")
    buf[0, 0, :, :W] = cuda32(r0)
    buf[1, 0, :, :W] = cuda32(r1)
    cfg = L.make_config(sweeps_per_pass=depth)
    L.check(L.lib().hs_matrix_powers(float(lam), D.ptr(Ixd), D.ptr(Iyd), D.ptr(buf[0, 0]),
                                     D.ptr(buf[1, 0]), H, W, ld, steps, D.ptr(buf[0, 0]),
                                     D.ptr(buf[1, 0]), H * ld, ctypes.byref(cfg),
                                     D.stream_handle()), "hs_matrix_powers")
    torch.cuda.synchronize()
    for s in range(steps):
        assert_bitexact(buf[0, s, :, :W].cpu().numpy(), R0[s], f"V0[{s}]")
        assert_bitexact(buf[1, s, :, :W].cpu().numpy(), R1[s], f"V1[{s}]")


def test_matrix_powers_single_step_is_copy(cuda):
    rng = np.random.default_rng(1)
    a = [rng.standard_normal((9, 11)).astype(np.float32) for _ in range(4)]
    V0, V1 = cg.hs_matrix_powers(1.0, *(cuda32(x) for x in a), 1)
    assert V0.shape == (1, 9, 11)
    assert_bitexact(V0[0].cpu().numpy(), a[2])
    assert_bitexact(V1[0].cpu().numpy(), a[3])


@pytest.mark.parametrize("name", ["precond_rand", "precond_zero"])
def test_preconditioner_reference_golden(cuda, name):
    g = golden(name + ".npz")
    for i in range(int(g["n"])):
        y0, y1 = cg.apply_hs_preconditioner(float(g["s2"]), *(cuda32(g[f"{k}_{i}"]) for k in ("d0", "d1", "od", "x0", "x1")))
        torch.cuda.synchronize()
        assert_bitexact(y0.cpu().numpy(), g[f"y0_{i}"])
        assert_bitexact(y1.cpu().numpy(), g[f"y1_{i}"])


def test_preconditioner_against_reference_template_golden(cuda):
    """ApplyHSPreconditioner's device template run as C, with determinants at, just below and
    at minus float(1e-15) (compared in double, as the template does): bit-identical."""
    g = golden("tmpl_precond.npz")
    for i in range(int(g["n"])):
        y0, y1 = cg.apply_hs_preconditioner(float(g[f"s2_{i}"]), *(cuda32(g[f"{k}_{i}"]) for k in ("d0", "d1", "od", "x0", "x1")))
        torch.cuda.synchronize()
        assert_bitexact(y0.cpu().numpy(), g[f"y0_{i}"], f"case {i}")
        assert_bitexact(y1.cpu().numpy(), g[f"y1_{i}"], f"case {i}")


def test_preconditioner_bitexact_with_singular_blocks(cuda):
    rng = np.random.default_rng(4)
    H, W = 37, 53
    d0 = rng.uniform(-1, 1, (H, W)).astype(np.float32)
    d1 = rng.uniform(-1, 1, (H, W)).astype(np.float32)
    od = rng.uniform(-1, 1, (H, W)).astype(np.float32)
    d0[::3, ::4] = 0.0
    d1[::3, ::4] = 0.0
    od[::3, ::4] = 0.0  # det = 0 there when s2 = 0
    x0, x1 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(2))
    for s2 in (0.0, 0.3):
        y0, y1 = cg.apply_hs_preconditioner(s2, *(cuda32(a) for a in (d0, d1, od, x0, x1)))
        r0, r1 = O.c_apply_hs_precond(s2, d0, d1, od, x0, x1)
        assert_bitexact(y0.cpu().numpy(), r0)
        assert_bitexact(y1.cpu().numpy(), r1)


def test_pcg_solves_hs_system(cuda):
    import scipy.sparse.linalg as spla

    from hindemith_b200 import synthetic
    I0, I1, _, _ = synthetic.make_pair(48, 64, 77)
    Ix, Iy, It = O.c_hs_derivs(I0, I1)
    alpha = 0.5
    u, v, res = cg.hs_pcg(cuda32(Ix), cuda32(Iy), cuda32(It), alpha, 400)
    torch.cuda.synchronize()
    M = O.hs_normal_matrix(alpha * alpha, Ix, Iy)
    b = -np.concatenate([(Ix.astype(np.float64) * It).ravel(), (Iy.astype(np.float64) * It).ravel()])
    w = spla.spsolve(M.tocsc(), b)
    got = np.concatenate([u.cpu().numpy().ravel(), v.cpu().numpy().ravel()]).astype(np.float64)
    assert float(res[-1]) < 1e-4
    assert np.abs(got - w).max() <= 1e-3 * np.abs(w).max()
