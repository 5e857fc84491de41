"""The fused mean end-point-error loss (hs_epe_loss_batched and its backward) against a
float64 PyTorch reference.  Tolerance: 1e-6 relative on the loss, 1e-5 on the gradients."""
import numpy as np
import pytest
import torch

from hindemith_b200 import _lib as L
from hindemith_b200.loss import mean_epe_batch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shapes", [[(1, 1)], [(5, 7), (64, 64)], [(37, 130)] * 3 + [(256, 300)]])
def test_mean_epe_batch_matches_float64(cuda, shapes):
    rng = np.random.default_rng(len(shapes))
    flows, targets, f64, t64 = [], [], [], []
    for H, W in shapes:
        a = [rng.standard_normal((H, W)).astype(np.float32) for _ in range(4)]
        flows.append(tuple(torch.from_numpy(x).cuda().requires_grad_(True) for x in a[:2]))
        targets.append(tuple(torch.from_numpy(x).cuda() for x in a[2:]))
        f64.append(tuple(torch.tensor(x, dtype=torch.float64, requires_grad=True) for x in a[:2]))
        t64.append(tuple(torch.tensor(x, dtype=torch.float64) for x in a[2:]))
    loss = mean_epe_batch(flows, targets)
    (2.5 * loss).backward()
    torch.cuda.synchronize()
    ref = sum(torch.sqrt((u - ut) ** 2 + (v - vt) ** 2 + 1e-12).mean()
              for (u, v), (ut, vt) in zip(f64, t64)) / len(f64)
    (2.5 * ref).backward()
    assert abs(float(loss.detach()) - float(ref.detach())) <= 1e-6 * abs(float(ref.detach()))
    for (u, v), (ur, vr) in zip(flows, f64):
        for g, r in ((u.grad, ur.grad), (v.grad, vr.grad)):
            err = np.abs(g.cpu().numpy() - r.numpy()).max() / np.abs(r.numpy()).max()
            assert err < 1e-5


def test_mean_epe_batch_deterministic(cuda):
    rng = np.random.default_rng(3)
    a = [torch.from_numpy(rng.standard_normal((300, 257)).astype(np.float32)).cuda() for _ in range(4)]
    l1 = mean_epe_batch([(a[0], a[1])], [(a[2], a[3])])
    l2 = mean_epe_batch([(a[0], a[1])], [(a[2], a[3])])
    assert float(l1) == float(l2)


def test_epe_argument_checks(cuda):
    lib = L.lib()
    d = (L.hs_epe_pair * 1)()
    assert lib.hs_epe_loss_batched(d, 1, 1e-12, None, None, 0, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_epe_workspace_bytes(0) == 0 and lib.hs_epe_workspace_bytes(33) == 0
