"""Gradients of the differentiable Horn-Schunck (hs_forward_train + hs_backward through
torch.autograd) against the FP64 reverse-mode oracle, a pure-PyTorch float64 autograd
reference and FP64 central finite differences.  Tolerance: 1e-3 relative (FP32
gradients against FP64 references)."""
import numpy as np
import pytest
import torch

from conftest import assert_bitexact
from hindemith_b200 import _lib as L
from hindemith_b200 import device as D
from hindemith_b200 import synthetic
from hindemith_b200.autograd import horn_schunck
from hs_torch_ref import hs_torch, mean_epe
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

REL = 1e-3


def cuda32(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-6)


def run_grad(I0, I1, alpha, iters, lam_u, lam_v, ckpt_every=10, fast=False):
    a = torch.tensor(alpha, dtype=torch.float32, device="cuda", requires_grad=True)
    x0 = cuda32(I0).requires_grad_(True)
    x1 = cuda32(I1).requires_grad_(True)
    u, v = horn_schunck(x0, x1, a, iters, ckpt_every, L.make_config(fast_math=fast))
    loss = (u * cuda32(lam_u)).sum() + (v * cuda32(lam_v)).sum()
    loss.backward()
    torch.cuda.synchronize()
    return (x0.grad.cpu().numpy(), x1.grad.cpu().numpy(), float(a.grad), u.detach().cpu().numpy(),
            v.detach().cpu().numpy())


@pytest.mark.parametrize("shape,iters,ckpt", [((1, 1), 5, 2), ((2, 3), 9, 4), ((24, 31), 20, 7),
                                              ((33, 65), 30, 10), ((7, 130), 12, 12)])
def test_grad_matches_fp64_adjoint(cuda, shape, iters, ckpt):
    H, W = shape
    rng = np.random.default_rng(H * 100 + W)
    I0, I1, _, _ = synthetic.make_pair(H, W, seed=1000 + H)
    lam_u = rng.standard_normal((H, W))
    lam_v = rng.standard_normal((H, W))
    alpha = 0.9
    g0, g1, ga, u, v = run_grad(I0, I1, alpha, iters, lam_u, lam_v, ckpt)
    r0, r1, ra, (ru, rv) = O.hs_adjoint_f64(I0.astype(np.float64), I1.astype(np.float64), alpha,
                                            iters, lam_u, lam_v)
    assert rel_err(g0, r0) < REL and rel_err(g1, r1) < REL
    assert abs(ga - ra) <= REL * abs(ra) + 1e-6
    assert np.abs(u - ru).max() < 1e-4


def test_forward_train_equals_forward(cuda):
    I0, I1, _, _ = synthetic.make_pair(70, 130, seed=1234)
    a = torch.tensor(1.3, device="cuda")
    u, v = horn_schunck(cuda32(I0), cuda32(I1), a, 37, 10)
    ru, rv = D.hs_forward(D.as_plane(cuda32(I0)), D.as_plane(cuda32(I1)), 1.3, 37)
    torch.cuda.synchronize()
    assert_bitexact(u.cpu().numpy(), ru.cpu().numpy(), "u")
    assert_bitexact(v.cpu().numpy(), rv.cpu().numpy(), "v")


def test_grad_independent_of_checkpoint_interval(cuda):
    """The recomputed states equal the forward's bit for bit, so the checkpoint interval
    changes only how the adjoint passes group the gradient accumulations (each pass adds
    its partial sums once): gradients agree to FP32 rounding of those sums, and a given
    interval gives the same bits run after run."""
    I0, I1, _, _ = synthetic.make_pair(40, 52, seed=77)
    rng = np.random.default_rng(1)
    lam_u, lam_v = rng.standard_normal((40, 52)), rng.standard_normal((40, 52))
    ref = run_grad(I0, I1, 1.1, 23, lam_u, lam_v, ckpt_every=23)
    for c in (1, 4, 10, 50):
        got = run_grad(I0, I1, 1.1, 23, lam_u, lam_v, ckpt_every=c)
        again = run_grad(I0, I1, 1.1, 23, lam_u, lam_v, ckpt_every=c)
        for a, b, n in ((got[0], again[0], "dI0"), (got[1], again[1], "dI1")):
            assert_bitexact(a, b, f"{n} rerun ckpt_every={c}")
        assert got[2] == again[2]
        assert rel_err(got[0], ref[0]) < 1e-5 and rel_err(got[1], ref[1]) < 1e-5, c
        assert abs(got[2] - ref[2]) <= 1e-5 * abs(ref[2]), c
        assert_bitexact(got[3], ref[3], f"u ckpt_every={c}")


def test_grad_epe_against_torch_autograd(cuda):
    """Config-3 style: 64x64 crop, 200 sweeps, checkpoint every 10, mean EPE loss."""
    I0, I1, ut, vt = synthetic.make_pair(64, 64, seed=1000)
    a = torch.tensor(1.0, device="cuda", requires_grad=True)
    x0 = cuda32(I0).requires_grad_(True)
    x1 = cuda32(I1).requires_grad_(True)
    u, v = horn_schunck(x0, x1, a, 200, 10)
    mean_epe(u, v, cuda32(ut), cuda32(vt)).backward()
    t0 = torch.from_numpy(I0.astype(np.float64)).requires_grad_(True)
    t1 = torch.from_numpy(I1.astype(np.float64)).requires_grad_(True)
    ta = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    ru, rv = hs_torch(t0, t1, ta, 200)
    mean_epe(ru, rv, torch.from_numpy(ut.astype(np.float64)),
             torch.from_numpy(vt.astype(np.float64))).backward()
    assert rel_err(x0.grad.cpu().numpy(), t0.grad.numpy()) < REL
    assert rel_err(x1.grad.cpu().numpy(), t1.grad.numpy()) < REL
    assert abs(float(a.grad) - float(ta.grad)) <= REL * abs(float(ta.grad))


def test_grad_finite_differences_fp64(cuda):
    """FP64 central differences of the mean-EPE loss on a 64x64 crop (the oracle's FP64
    forward) at the pixels with the largest gradients, and for alpha."""
    I0, I1, ut, vt = synthetic.make_pair(64, 64, seed=1001)
    iters, alpha = 60, 1.0
    a = torch.tensor(alpha, device="cuda", requires_grad=True)
    x0 = cuda32(I0).requires_grad_(True)
    x1 = cuda32(I1).requires_grad_(True)
    u, v = horn_schunck(x0, x1, a, iters, 10)
    mean_epe(u, v, cuda32(ut), cuda32(vt)).backward()
    g0, g1, ga = x0.grad.cpu().numpy(), x1.grad.cpu().numpy(), float(a.grad)

    U, V = ut.astype(np.float64), vt.astype(np.float64)

    def loss(i0, i1, al):
        uu, vv = O.c_hs_forward(i0, i1, al, iters, np.float64)
        return np.sqrt((uu - U) ** 2 + (vv - V) ** 2 + 1e-12).mean()

    b0, b1 = I0.astype(np.float64), I1.astype(np.float64)
    h = 1e-4
    for g, which in ((g0, 0), (g1, 1)):
        for flat in np.argsort(-np.abs(g).ravel())[:4]:
            i, j = divmod(int(flat), g.shape[1])
            p, m = (b0.copy(), b1.copy()), (b0.copy(), b1.copy())
            p[which][i, j] += h
            m[which][i, j] -= h
            fd = (loss(*p, alpha) - loss(*m, alpha)) / (2 * h)
            assert abs(g[i, j] - fd) <= REL * abs(fd), (which, i, j, g[i, j], fd)
    fda = (loss(b0, b1, alpha + h) - loss(b0, b1, alpha - h)) / (2 * h)
    assert abs(ga - fda) <= REL * abs(fda), (ga, fda)


def test_grad_fast_form(cuda):
    I0, I1, _, _ = synthetic.make_pair(33, 65, seed=5)
    rng = np.random.default_rng(2)
    lam_u, lam_v = rng.standard_normal((33, 65)), rng.standard_normal((33, 65))
    g0, g1, ga, _, _ = run_grad(I0, I1, 0.7, 25, lam_u, lam_v, 10, fast=True)
    r0, r1, ra, _ = O.hs_adjoint_f64(I0.astype(np.float64), I1.astype(np.float64), 0.7, 25,
                                     lam_u, lam_v)
    assert rel_err(g0, r0) < REL and rel_err(g1, r1) < REL
    assert abs(ga - ra) <= REL * abs(ra)


# ---------------------------------------------------------------- batched training path

def run_batch_grad(imgs, alpha, iters, lams, ckpt_every=10, T=4, fast=True, layout=0):
    from hindemith_b200.autograd import horn_schunck_batch

    a = torch.tensor(alpha, dtype=torch.float32, device="cuda", requires_grad=True)
    xs = [(cuda32(I0).requires_grad_(True), cuda32(I1).requires_grad_(True)) for I0, I1 in imgs]
    outs = horn_schunck_batch(xs, a, iters, ckpt_every,
                              L.make_config(sweeps_per_pass=T, fast_math=fast, layout=layout))
    loss = 0
    for (u, v), (lu, lv) in zip(outs, lams):
        loss = loss + (u * cuda32(lu)).sum() + (v * cuda32(lv)).sum()
    loss.backward()
    torch.cuda.synchronize()
    return ([(x0.grad.cpu().numpy(), x1.grad.cpu().numpy()) for x0, x1 in xs], float(a.grad),
            [(u.detach().cpu().numpy(), v.detach().cpu().numpy()) for u, v in outs])


@pytest.mark.parametrize("T", [1, 3, 4, 5])
@pytest.mark.parametrize("ckpt", [1, 7, 10])
def test_batched_grad_matches_fp64_adjoint(cuda, T, ckpt):
    shapes = [(24, 31), (33, 65), (1, 9), (70, 130)]
    iters, alpha = 23, 0.8
    rng = np.random.default_rng(T * 10 + ckpt)
    imgs = [synthetic.make_pair(H, W, seed=500 + i)[:2] for i, (H, W) in enumerate(shapes)]
    lams = [(rng.standard_normal(s), rng.standard_normal(s)) for s in shapes]
    grads, ga, outs = run_batch_grad(imgs, alpha, iters, lams, ckpt, T)
    ra_total = 0.0
    for (I0, I1), (lu, lv), (g0, g1), (u, v) in zip(imgs, lams, grads, outs):
        r0, r1, ra, (ru, rv) = O.hs_adjoint_f64(I0.astype(np.float64), I1.astype(np.float64),
                                                alpha, iters, lu, lv)
        ra_total += ra
        assert rel_err(g0, r0) < REL and rel_err(g1, r1) < REL
        assert np.abs(u - ru).max() < 1e-4
    assert abs(ga - ra_total) <= REL * abs(ra_total)


@pytest.mark.parametrize("T", [3, 5])
def test_batched_grad_wide_layout_identical(cuda, T):
    """The training passes (forward and dump recompute) in the 4-columns-per-lane layout
    compute every cell as the 2-column ones: flows and gradients identical bit for bit."""
    shapes = [(70, 130), (33, 260), (1, 9)]
    rng = np.random.default_rng(T)
    imgs = [synthetic.make_pair(H, W, seed=700 + i)[:2] for i, (H, W) in enumerate(shapes)]
    lams = [(rng.standard_normal(s), rng.standard_normal(s)) for s in shapes]
    g1, a1, o1 = run_batch_grad(imgs, 0.9, 23, lams, 7, T, layout=1)
    g2, a2, o2 = run_batch_grad(imgs, 0.9, 23, lams, 7, T, layout=2)
    for (x0, x1), (y0, y1), (u1, v1), (u2, v2) in zip(g1, g2, o1, o2):
        assert_bitexact(y0, x0, "dI0")
        assert_bitexact(y1, x1, "dI1")
        assert_bitexact(u2, u1, "u")
        assert_bitexact(v2, v1, "v")
    assert a1 == a2


def test_batched_train_forward_equals_forward(cuda):
    from hindemith_b200.autograd import horn_schunck_batch

    imgs = [synthetic.make_pair(H, W, seed=9 + H)[:2] for H, W in ((64, 80), (17, 23))]
    a = torch.tensor(1.2, device="cuda")
    cfg = L.make_config(sweeps_per_pass=4)
    outs = horn_schunck_batch([(cuda32(x), cuda32(y)) for x, y in imgs], a, 37, 10, cfg)
    for (u, v), (I0, I1) in zip(outs, imgs):
        ru, rv = D.hs_forward(D.as_plane(cuda32(I0)), D.as_plane(cuda32(I1)), 1.2, 37, cfg)
        torch.cuda.synchronize()
        assert_bitexact(u.cpu().numpy(), ru.cpu().numpy(), "u")
        assert_bitexact(v.cpu().numpy(), rv.cpu().numpy(), "v")


def test_batched_grad_epe_config3_crop(cuda):
    """Four 64x64 crops, 200 sweeps, checkpoints every 10, mean EPE: against torch float64."""
    from hindemith_b200.autograd import horn_schunck_batch

    data = [synthetic.make_pair(64, 64, seed=1000 + i) for i in range(4)]
    a = torch.tensor(1.0, device="cuda", requires_grad=True)
    xs = [(cuda32(d[0]).requires_grad_(True), cuda32(d[1]).requires_grad_(True)) for d in data]
    outs = horn_schunck_batch(xs, a, 200, 10, L.make_config(sweeps_per_pass=4, fast_math=True))
    loss = sum(mean_epe(u, v, cuda32(d[2]), cuda32(d[3])) for (u, v), d in zip(outs, data)) / 4
    loss.backward()
    ta = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    tx = [(torch.from_numpy(d[0].astype(np.float64)).requires_grad_(True),
           torch.from_numpy(d[1].astype(np.float64)).requires_grad_(True)) for d in data]
    tl = 0
    for (t0, t1), d in zip(tx, data):
        ru, rv = hs_torch(t0, t1, ta, 200)
        tl = tl + mean_epe(ru, rv, torch.from_numpy(d[2].astype(np.float64)),
                           torch.from_numpy(d[3].astype(np.float64)))
    (tl / 4).backward()
    for (x0, x1), (t0, t1) in zip(xs, tx):
        assert rel_err(x0.grad.cpu().numpy(), t0.grad.numpy()) < REL
        assert rel_err(x1.grad.cpu().numpy(), t1.grad.numpy()) < REL
    assert abs(float(a.grad) - float(ta.grad)) <= REL * abs(float(ta.grad))
