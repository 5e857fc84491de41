"""The @hm drop-in on the GPU: the reference-surface programs against the golden
fixtures the reference's own NumPy library produced."""
import numpy as np
import pytest
import torch

import hs_programs
from conftest import assert_bitexact, golden, golden_files
from hindemith_b200 import Stencil, hm, hs_average_stencil, hs_derivative_stencils, state
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

Dx, Dy, Dt = hs_derivative_stencils()
A = hs_average_stencil()


def kwargs_for(d, **extra):
    z = np.zeros_like(d["I0"])
    kw = dict(I0=d["I0"], I1=d["I1"], Dx=Dx, Dy=Dy, Dt=Dt, A=A, u=z, v=z)
    kw.update(extra)
    return kw


@pytest.mark.parametrize("path", golden_files("hs_*.npz"))
def test_hm_hs_jacobi_golden(cuda, path):
    d = np.load(path)
    f = hm(hs_programs.hs_jacobi)
    u, v = f(**kwargs_for(d, alpha2=np.float32(d["alpha2"]), sweeps=np.int64(d["sweeps"])))
    assert isinstance(u, np.ndarray) and u.dtype == np.float32
    assert state["last_stats"]["hs_sweeps_calls"] == 1
    assert_bitexact(u, d["u"], "u")
    assert_bitexact(v, d["v"], "v")


def test_hm_literal_bound_program(cuda):
    d = golden("hs_24x31.npz")
    alpha = np.float32(1.3)
    f = hm(hs_programs.hs_jacobi_20)
    u, v = f(**kwargs_for(d, alpha=alpha))
    Ix, Iy, It = O.hs_derivs(d["I0"], d["I1"])
    z = np.zeros_like(d["I0"])
    ru, rv = O.hs_sweeps(Ix, Iy, It, alpha * alpha, 20, z, z)
    assert_bitexact(u, ru, "u")
    assert_bitexact(v, rv, "v")


@pytest.mark.parametrize("prog", [hs_programs.hs_jacobi_commuted, hs_programs.hs_jacobi_reassociated])
def test_hm_variants_match_their_numpy_meaning(cuda, prog):
    """Each program equals its own statement-by-statement FP32 meaning, fused or not."""
    from oracle.hs_oracle import stencil2d

    class NpStencil:  # the NumPy meaning of Stencil * Array2D (clamp-to-edge, tap order)
        def __init__(self, s):
            self.s = s

        def __mul__(self, x):
            return stencil2d(self.s.data, self.s.offx, self.s.offy, x)

    d = golden("hs_33x65.npz")
    z = np.zeros_like(d["I0"])
    kw = dict(I0=d["I0"], I1=d["I1"], alpha2=np.float32(d["alpha2"]), u=z, v=z, sweeps=13)
    ru, rv = prog(Dx=NpStencil(Dx), Dy=NpStencil(Dy), Dt=NpStencil(Dt), A=NpStencil(A), **kw)
    f = hm(prog)
    u, v = f(Dx=Dx, Dy=Dy, Dt=Dt, A=A, **dict(kw, sweeps=np.int64(13)))
    assert_bitexact(u, ru, "u")
    assert_bitexact(v, rv, "v")


def test_hm_torch_in_torch_out(cuda):
    d = golden("hs_70x130.npz")
    f = hm(hs_programs.hs_jacobi)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    z = torch.zeros(d["I0"].shape, device="cuda")
    u, v = f(I0=t(d["I0"]), I1=t(d["I1"]), Dx=Dx, Dy=Dy, Dt=Dt, A=A,
             alpha2=np.float32(d["alpha2"]), u=z, v=z, sweeps=np.int64(d["sweeps"]))
    assert isinstance(u, torch.Tensor) and u.is_cuda
    assert_bitexact(u.cpu().numpy(), d["u"], "u")


def test_hm_nonstandard_average_runs_unfused(cuda):
    """A 4-neighbour average is not the fused kernel's stencil: the loop runs one
    operator per statement and still matches its NumPy meaning."""
    A4 = Stencil(np.full(4, 0.25, np.float32), [-1, 1, 0, 0], [0, 0, -1, 1])
    d = golden("hs_24x31.npz")
    f = hm(hs_programs.hs_jacobi)
    kw = kwargs_for(d, alpha2=np.float32(d["alpha2"]), sweeps=np.int64(6))
    kw["A"] = A4
    u, v = f(**kw)
    assert state["last_stats"]["unfused_loops"] == 1
    Ix, Iy, It = O.hs_derivs(d["I0"], d["I1"])
    den = np.float32(d["alpha2"]) + Ix * Ix + Iy * Iy
    ru = rv = np.zeros_like(d["I0"])
    for _ in range(6):
        ub = O.stencil2d(A4.data, A4.offx, A4.offy, ru)
        vb = O.stencil2d(A4.data, A4.offx, A4.offy, rv)
        t = (Ix * ub + Iy * vb + It) / den
        ru, rv = ub - Ix * t, vb - Iy * t
    assert_bitexact(u, ru, "u")
    assert_bitexact(v, rv, "v")


def test_stencil_mul_outside_hm(cuda):
    d = np.load(golden_files("stencil_avg.npz")[0])
    x = d["x4"]
    y = A * x
    assert isinstance(y, np.ndarray)
    assert_bitexact(y, d["out4"], "A*x")


@pytest.mark.parametrize("fast", [False, True])
def test_hm_without_defines_runs_the_tuned_sweep(cuda, fast):
    """With no depth in `defines`, the fused loop runs the configuration the autotuner picks
    for the shape and form; the exact form stays bit-identical to the golden fixture, the
    fast form within 1e-4 of it."""
    from hindemith_b200 import autotune
    from hindemith_b200 import defines

    d = golden("hs_70x130.npz")
    old = dict(defines)
    try:
        defines.clear()
        if fast:
            defines["hs_fast_math"] = True
        f = hm(hs_programs.hs_jacobi)
        u, v = f(**kwargs_for(d, alpha2=np.float32(d["alpha2"]), sweeps=np.int64(d["sweeps"])))
        ex = next(iter(f._cache.values()))
    finally:
        defines.clear()
        defines.update(old)
    H, W = d["I0"].shape
    T, seg, layout = autotune.best_sweep_config(H, W, (W + 3) // 4 * 4, fast_math=fast)
    assert ex.last_sweep_config == (T, seg, layout, fast)
    if fast:
        assert np.abs(u - d["u"]).max() < 1e-4 and np.abs(v - d["v"]).max() < 1e-4
    else:
        assert_bitexact(u, d["u"], "u")
        assert_bitexact(v, d["v"], "v")
