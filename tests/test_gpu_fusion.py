"""Generic @hm programs through the fused, runtime-compiled kernels: every program must
equal its own statement-by-statement FP32 meaning (NumPy float32 arithmetic, the oracle's
clamp-to-edge stencil, double-accumulated sum2d rounded once), fused or not."""
import numpy as np
import pytest

from conftest import assert_bitexact
from hindemith_b200 import Stencil, hm, hs_average_stencil, hs_derivative_stencils, state
from hindemith_b200 import hindemith as HM
from oracle.hs_oracle import stencil2d

pytestmark = pytest.mark.gpu


# ---- the NumPy meaning of the surface's calls (used when a program runs as plain Python)
def sqrt(x):
    return np.sqrt(x) if isinstance(x, np.ndarray) else np.float32(np.sqrt(np.float32(x)))


def sum2d(x):
    return np.float32(np.sum(x.astype(np.float64)))


def red(x):
    Y, X = np.indices(x.shape)
    return np.where((X + Y) & 1, np.float32(0.0), x).astype(np.float32)


def black(x):
    Y, X = np.indices(x.shape)
    return np.where((X + Y) & 1, x, np.float32(0.0)).astype(np.float32)


class NpStencil:
    def __init__(self, s):
        self.s = s

    def __mul__(self, x):
        return stencil2d(self.s.data, self.s.offx, self.s.offy, x)


def np_meaning(fn, **kw):
    conv = {k: (NpStencil(v) if isinstance(v, Stencil) else v) for k, v in kw.items()}
    with np.errstate(divide="ignore", invalid="ignore"):
        return fn(**conv)


# ---- programs
def grad_magnitude(I0, I1, Dx, Dy, Dt):
    Ix = Dx * I0 + Dx * I1
    Iy = Dy * I0 + Dy * I1
    It = Dt * I1 - Dt * I0
    m = sqrt(Ix * Ix + Iy * Iy + 0.001)
    s = sum2d(m)
    n = m / s
    return n, It, s


def red_black_mix(x, A, w):
    r = red(x) + w * black(A * x)
    t = black(r) - red(A * r)
    return t


def smooth_loop(x, A, k, beta):
    u = x
    for i in range(k):
        u = A * u + beta * x
    return u, sum2d(u * u)


def chain_with_scalar_between(x, y, a, A2):
    p = x * y
    b = a * 2.0 + 1.0
    q = p / b - x
    r = A2 * q
    return r, p


def two_outputs(x, y):
    u = x + y
    v = x - y
    w = u * v
    return w, u


Dx, Dy, Dt = hs_derivative_stencils()
A = hs_average_stencil()


@pytest.fixture(params=[True, False], ids=["fused", "unfused"])
def fuse(request):
    old = dict(HM.defines)
    HM.defines["hs_fuse"] = request.param
    yield request.param
    HM.defines.clear()
    HM.defines.update(old)


def rnd(shape, seed, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, shape).astype(np.float32)


@pytest.mark.parametrize("shape", [(1, 1), (7, 5), (64, 96), (131, 257)])
def test_grad_magnitude(cuda, fuse, shape):
    I0, I1 = rnd(shape, 1), rnd(shape, 2)
    got = hm(grad_magnitude)(I0=I0, I1=I1, Dx=Dx, Dy=Dy, Dt=Dt)
    want = np_meaning(grad_magnitude, I0=I0, I1=I1, Dx=Dx, Dy=Dy, Dt=Dt)
    assert abs(float(got[2]) - float(want[2])) <= 1e-6 * abs(float(want[2]))
    assert_bitexact(got[1], want[1], "It")
    # n = m / s uses the device sum, which may differ from the host's in the last bit
    np.testing.assert_allclose(got[0], want[0], rtol=2e-7, atol=0)
    if fuse:
        assert state["last_stats"]["fused_launches"] == 2


@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (33, 65)])
def test_red_black_and_stencil_split(cuda, fuse, shape):
    x = rnd(shape, 3)
    w = np.float32(0.37)
    got = hm(red_black_mix)(x=x, A=A, w=w)
    want = np_meaning(red_black_mix, x=x, A=A, w=w)
    assert_bitexact(got, want)
    if fuse:  # A * r reads r, written in the same group: the group splits there
        assert state["last_stats"]["fused_launches"] == 2


def test_loop_carried_values(cuda, fuse):
    x = rnd((40, 50), 4)
    got = hm(smooth_loop)(x=x, A=A, k=np.int64(6), beta=np.float32(0.25))
    want = np_meaning(smooth_loop, x=x, A=A, k=6, beta=np.float32(0.25))
    assert_bitexact(got[0], want[0])
    assert abs(float(got[1]) - float(want[1])) <= 1e-6 * abs(float(want[1]))


def test_scalar_statements_between_array_statements(cuda, fuse):
    x, y = rnd((17, 23), 5), rnd((17, 23), 6, 0.5, 2.0)
    kw = dict(x=x, y=y, a=np.float32(1.5), A2=A)
    got = hm(chain_with_scalar_between)(**kw)
    want = np_meaning(chain_with_scalar_between, **kw)
    assert_bitexact(got[0], want[0])
    assert_bitexact(got[1], want[1])


def test_dead_intermediates_stay_in_registers(cuda):
    from hindemith_b200.frontend import parse
    from hindemith_b200.fusion import fuse_program

    x, y = rnd((9, 9), 7), rnd((9, 9), 8)
    got = hm(two_outputs)(x=x, y=y)
    want = np_meaning(two_outputs, x=x, y=y)
    assert_bitexact(got[0], want[0])
    assert_bitexact(got[1], want[1])
    prog = parse(HM.function_source(two_outputs), {"x": "Array2D", "y": "Array2D"})
    fuse_program(prog)
    fused = [s for s in prog.body if s.kind == "Fused"]
    assert len(fused) == 1
    assert set(fused[0].info["outputs"]) == {"w", "u"}  # v is dead after the group


def echo_and_repeat(x, y, A2):
    s = A2 * x
    t = s + y
    return x, s, t, s


def test_results_never_alias_arguments_or_each_other(cuda, fuse):
    """Values the call computed come back as they are; an argument, or a value returned twice,
    comes back as a copy: writing one result changes no argument and no other result."""
    import torch

    x = torch.from_numpy(rnd((37, 45), 9)).cuda()
    y = torch.from_numpy(rnd((37, 45), 10)).cuda()
    x0 = x.clone()
    got = hm(echo_and_repeat)(x=x, y=y, A2=A)
    want = np_meaning(echo_and_repeat, x=x0.cpu().numpy(), y=y.cpu().numpy(), A2=A)
    for g, w in zip(got, want):
        assert_bitexact(g.cpu().numpy(), w)
    for g in got:
        g.fill_(123.0)
        assert torch.equal(x, x0)
    for i, g in enumerate(got):
        g.fill_(float(i))
        for j, h in enumerate(got[:i]):
            assert bool((h == float(j)).all()), (i, j)
