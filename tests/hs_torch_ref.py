"""Pure-PyTorch Horn-Schunck (test reference for gradients): clamp-to-edge stencils via
replicate padding, autograd does the reverse mode.  Float64 by default."""
import torch
import torch.nn.functional as F

AVG = torch.tensor([[1 / 12, 1 / 6, 1 / 12], [1 / 6, 0.0, 1 / 6], [1 / 12, 1 / 6, 1 / 12]])
DX = torch.tensor([[-0.25, 0.25], [-0.25, 0.25]])
DY = torch.tensor([[-0.25, -0.25], [0.25, 0.25]])
DT = torch.tensor([[0.25, 0.25], [0.25, 0.25]])


def _conv(x, k, pad):
    # x (H, W); pad = (left, right, top, bottom) with edge replication, then correlation
    y = F.pad(x[None, None], pad, mode="replicate")
    return F.conv2d(y, k.to(x)[None, None])[0, 0]


def hs_torch(I0, I1, alpha, iters):
    Ix = _conv(I0, DX, (0, 1, 0, 1)) + _conv(I1, DX, (0, 1, 0, 1))
    Iy = _conv(I0, DY, (0, 1, 0, 1)) + _conv(I1, DY, (0, 1, 0, 1))
    It = _conv(I1, DT, (0, 1, 0, 1)) - _conv(I0, DT, (0, 1, 0, 1))
    d = alpha * alpha + Ix * Ix + Iy * Iy
    u = torch.zeros_like(I0)
    v = torch.zeros_like(I0)
    for _ in range(iters):
        ub = _conv(u, AVG, (1, 1, 1, 1))
        vb = _conv(v, AVG, (1, 1, 1, 1))
        t = (Ix * ub + Iy * vb + It) / d
        u, v = ub - Ix * t, vb - Iy * t
    return u, v


def mean_epe(u, v, ut, vt, eps=1e-12):
    return torch.sqrt((u - ut) ** 2 + (v - vt) ** 2 + eps).mean()
