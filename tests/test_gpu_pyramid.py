"""Coarse-to-fine pieces (hs_blur_down, hs_upsample2, hs_warp and their adjoints) against
the FP64 oracle and the FP32 warp restatement, and the differentiable coarse-to-fine
pipeline against a float64 PyTorch autograd reference.  Tolerances: the warp is
bit-identical to the reference's float/double arithmetic; the linear maps agree with
FP64 to 1e-6 relative; pipeline flows to 1e-4 max-abs and gradients to 1e-3 relative."""
import numpy as np
import pytest
import torch

from conftest import golden
from hindemith_b200 import _lib as L
from hindemith_b200 import pyramid as PY
from hindemith_b200 import synthetic
from hs_torch_ref import coarse_to_fine_torch, mean_epe
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 3), (5, 4), (37, 53), (64, 64), (130, 97)]


def cuda32(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def _bits32(a):
    """The float32 bit patterns of a (any shape, 0-d included)."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32)).reshape(-1).view(np.uint32)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-6)


@pytest.mark.parametrize("shape", SHAPES)
def test_blur_down_and_adjoint(cuda, shape):
    H, W = shape
    rng = np.random.default_rng(H * 131 + W)
    x = rng.standard_normal((H, W)).astype(np.float32)
    g = rng.standard_normal(((H + 1) // 2, (W + 1) // 2)).astype(np.float32)
    xt = cuda32(x).requires_grad_(True)
    y = PY.blur_down(xt)
    y.backward(cuda32(g))
    torch.cuda.synchronize()
    assert rel_err(host(y), O.blur_down(x)) < 1e-6
    assert rel_err(host(xt.grad), O.blur_down_adjoint(g, H, W)) < 1e-6


@pytest.mark.parametrize("shape", SHAPES)
def test_upsample2_and_adjoint(cuda, shape):
    H, W = shape
    Hc, Wc = (H + 1) // 2, (W + 1) // 2
    rng = np.random.default_rng(H * 71 + W)
    c = rng.standard_normal((Hc, Wc)).astype(np.float32)
    g = rng.standard_normal((H, W)).astype(np.float32)
    ct = cuda32(c).requires_grad_(True)
    f = PY.upsample2(ct, H, W, 2.0)
    f.backward(cuda32(g))
    torch.cuda.synchronize()
    assert rel_err(host(f), O.upsample2(c, H, W, 2.0)) < 1e-6
    assert rel_err(host(ct.grad), O.upsample2_adjoint(g, Hc, Wc, 2.0)) < 1e-6


@pytest.mark.parametrize("shape,amp", [((1, 1), 0.5), ((7, 9), 3.0), ((64, 80), 2.5),
                                       ((129, 257), 12.0)])
def test_warp_bitexact(cuda, shape, amp):
    H, W = shape
    rng = np.random.default_rng(H + 7 * W)
    src = rng.random((H, W)).astype(np.float32)
    ox = rng.uniform(-amp, amp, (H, W)).astype(np.float32)
    oy = rng.uniform(-amp, amp, (H, W)).astype(np.float32)
    # integer and negative-integer offsets take the reference's truncate-then-step rule
    ox.flat[::7] = np.round(ox.flat[::7])
    oy.flat[::5] = np.round(oy.flat[::5])
    out = PY.warp(cuda32(src), cuda32(ox), cuda32(oy))
    torch.cuda.synchronize()
    ref = O.c_warp(src, ox, oy)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_warp_against_reference_template_golden(cuda):
    """hs_warp against the reference's WarpImg2D device template run as C: bit-identical."""
    g = golden("tmpl_warp.npz")
    for i in range(int(g["n"])):
        out = PY.warp(cuda32(g[f"src_{i}"]), cuda32(g[f"ox_{i}"]), cuda32(g[f"oy_{i}"]))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), g[f"out_{i}"].view(np.uint32))


def test_warp_adjoint(cuda):
    H, W = 70, 91
    rng = np.random.default_rng(5)
    src = rng.random((H, W)).astype(np.float32)
    ox = rng.uniform(-4, 4, (H, W)).astype(np.float32)
    oy = rng.uniform(-4, 4, (H, W)).astype(np.float32)
    g = rng.standard_normal((H, W)).astype(np.float32)
    s, u, v = (cuda32(a).requires_grad_(True) for a in (src, ox, oy))
    PY.warp(s, u, v).backward(cuda32(g))
    torch.cuda.synchronize()
    ds, du, dv = O.warp_adjoint_f64(src, ox, oy, g)
    assert rel_err(host(s.grad), ds) < 1e-5
    assert rel_err(host(u.grad), du) < 1e-5
    assert rel_err(host(v.grad), dv) < 1e-5


@pytest.mark.parametrize("gscale", [1.0, 1e-9])
def test_warp_adjoint_deterministic(cuda, gscale):
    """dL/dsrc is summed in fixed point: a contracting flow that sends many destination
    pixels into the same source footprints gives the same bits run after run, and stays
    within 1e-5 of FP64 at any gradient magnitude."""
    H, W = 130, 257
    rng = np.random.default_rng(9)
    src = rng.random((H, W)).astype(np.float32)
    Y, X = np.mgrid[0:H, 0:W].astype(np.float32)
    ox = (0.3 * (W / 2 - X) + rng.uniform(-0.5, 0.5, (H, W))).astype(np.float32)
    oy = (0.3 * (H / 2 - Y) + rng.uniform(-0.5, 0.5, (H, W))).astype(np.float32)
    g = (gscale * rng.standard_normal((H, W))).astype(np.float32)
    grads = []
    for _ in range(3):
        s, u, v = (cuda32(a).requires_grad_(True) for a in (src, ox, oy))
        PY.warp(s, u, v).backward(cuda32(g))
        torch.cuda.synchronize()
        grads.append(host(s.grad))
    for a in grads[1:]:
        np.testing.assert_array_equal(a.view(np.uint32), grads[0].view(np.uint32))
    ds, _, _ = O.warp_adjoint_f64(src, ox, oy, g)
    assert rel_err(grads[0], ds) < 1e-5


def test_warp_adjoint_nonfinite_gradient_gives_nan(cuda):
    H, W = 16, 20
    src = np.ones((H, W), np.float32)
    z = np.zeros((H, W), np.float32)
    g = np.ones((H, W), np.float32)
    g[3, 4] = np.inf
    s, u, v = (cuda32(a).requires_grad_(True) for a in (src, z, z))
    PY.warp(s, u, v).backward(cuda32(g))
    torch.cuda.synchronize()
    assert np.isnan(host(s.grad)).all()


def test_pyramid_argument_errors(cuda):
    with pytest.raises(ValueError):
        PY.upsample2(torch.zeros((3, 3), device="cuda"), 8, 8)
    with pytest.raises(ValueError):
        PY.warp(torch.zeros((4, 4), device="cuda"), torch.zeros((4, 5), device="cuda"),
                torch.zeros((4, 4), device="cuda"))
    lib = L.lib()
    x = torch.zeros((8, 8), device="cuda")
    # output row stride below the coarse width
    assert lib.hs_blur_down(x.data_ptr(), 8, 8, 8, x.data_ptr(), 2, None) == L.HS_ERR_INVALID_ARG


def _pairs(n, H, W, amp, seed=300):
    out = []
    for i in range(n):
        I0, I1, u, v = synthetic.make_pair(H, W, seed + i, sigma=2.0, amplitude=amp)
        out.append((I0, I1, u, v))
    return out


def test_coarse_to_fine_forward_matches_float64(cuda):
    data = _pairs(2, 96, 128, 5.0)
    pairs = [(cuda32(a), cuda32(b)) for a, b, _, _ in data]
    flows = PY.coarse_to_fine(pairs, 1.0, levels=3, iters=40, ckpt_every=10,
                              config=L.make_config(fast_math=0))
    torch.cuda.synchronize()
    for (I0, I1, _, _), (u, v) in zip(data, flows):
        ur, vr = coarse_to_fine_torch(torch.from_numpy(I0.astype(np.float64)),
                                      torch.from_numpy(I1.astype(np.float64)), 1.0, 3, 40)
        assert np.abs(host(u) - ur.numpy()).max() < 1e-4
        assert np.abs(host(v) - vr.numpy()).max() < 1e-4


@pytest.mark.parametrize("fast", [0, 1])
def test_coarse_to_fine_grad_matches_float64_autograd(cuda, fast):
    data = _pairs(2, 64, 80, 4.0, seed=410)
    levels, iters = 3, 30
    a = torch.tensor(1.0, device="cuda", requires_grad=True)
    xs = [(cuda32(I0).requires_grad_(True), cuda32(I1).requires_grad_(True))
          for I0, I1, _, _ in data]
    flows = PY.coarse_to_fine(xs, a, levels=levels, iters=iters, ckpt_every=10,
                              config=L.make_config(fast_math=fast))
    loss = sum(mean_epe(u, v, cuda32(ut), cuda32(vt))
               for (u, v), (_, _, ut, vt) in zip(flows, data)) / len(data)
    loss.backward()
    torch.cuda.synchronize()

    a64 = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    x64 = [(torch.tensor(I0, dtype=torch.float64, requires_grad=True),
            torch.tensor(I1, dtype=torch.float64, requires_grad=True)) for I0, I1, _, _ in data]
    loss64 = 0
    for (I0, I1), (_, _, ut, vt) in zip(x64, data):
        u, v = coarse_to_fine_torch(I0, I1, a64, levels, iters)
        loss64 = loss64 + mean_epe(u, v, torch.tensor(ut, dtype=torch.float64),
                                   torch.tensor(vt, dtype=torch.float64))
    (loss64 / len(data)).backward()

    assert abs(float(loss.detach()) - float(loss64) / len(data)) < 1e-5
    for (g0, g1), (r0, r1) in zip(xs, x64):
        assert rel_err(host(g0.grad), r0.grad.numpy()) < 1e-3
        assert rel_err(host(g1.grad), r1.grad.numpy()) < 1e-3
    assert abs(float(a.grad) - float(a64.grad)) <= 1e-3 * max(abs(float(a64.grad)), 1e-6)


def test_coarse_to_fine_graph_capture(cuda):
    """Forward + backward through all levels captured in one CUDA graph and replayed."""
    data = _pairs(2, 128, 128, 6.0, seed=520)
    I0s = [cuda32(I0) for I0, _, _, _ in data]
    I1s = [cuda32(I1) for _, I1, _, _ in data]
    uts = [(cuda32(u), cuda32(v)) for _, _, u, v in data]
    a = torch.tensor(1.0, device="cuda")
    cfg = L.make_config(fast_math=1)

    def step():
        # fresh leaves per call: an autograd leaf remembers the stream it was first used on
        al = a.detach().requires_grad_(True)
        xs = [(x0.detach().requires_grad_(True), x1.detach().requires_grad_(True))
              for x0, x1 in zip(I0s, I1s)]
        flows = PY.coarse_to_fine(xs, al, levels=3, iters=20, ckpt_every=10, config=cfg)
        loss = sum(mean_epe(u, v, ut, vt) for (u, v), (ut, vt) in zip(flows, uts)) / len(uts)
        grads = torch.autograd.grad(loss, [al] + [t for p in xs for t in p])
        return loss, grads

    eager_loss, eager_grads = step()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            step()
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        g_loss, g_grads = step()
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    assert abs(float(g_loss.detach()) - float(eager_loss.detach())) <= 1e-6 * abs(float(eager_loss.detach()))
    for x, y in zip(g_grads, eager_grads):
        # every adjoint is deterministic: the replay gives the eager bits
        np.testing.assert_array_equal(_bits32(host(x)), _bits32(host(y)))


def test_coarse_to_fine_gradients_are_bit_reproducible(cuda):
    """Every adjoint on the coarse-to-fine path is deterministic (gathers, fixed-order
    reductions, the fixed-point warp scatter): two backward passes give the same bits."""
    data = _pairs(2, 96, 112, 6.0, seed=610)
    runs = []
    for _ in range(2):
        a = torch.tensor(1.0, device="cuda", requires_grad=True)
        xs = [(cuda32(I0).requires_grad_(True), cuda32(I1).requires_grad_(True))
              for I0, I1, _, _ in data]
        flows = PY.coarse_to_fine(xs, a, levels=3, iters=20, ckpt_every=10,
                                  config=L.make_config(fast_math=1))
        loss = sum(mean_epe(u, v, cuda32(ut), cuda32(vt))
                   for (u, v), (_, _, ut, vt) in zip(flows, data)) / len(data)
        loss.backward()
        torch.cuda.synchronize()
        runs.append([host(t.grad) for p in xs for t in p] + [np.float32(a.grad.item())])
    for x, y in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(_bits32(x), _bits32(y))
