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


# ---------------------------------------------------------------- coarse-to-fine pieces

BIN5 = [1 / 16, 4 / 16, 6 / 16, 4 / 16, 1 / 16]


def blur_down_torch(x):
    H, W = x.shape
    Ho, Wo = (H + 1) // 2, (W + 1) // 2
    out = torch.zeros((Ho, Wo), dtype=x.dtype, device=x.device)
    ar_y = torch.arange(Ho, device=x.device)
    ar_x = torch.arange(Wo, device=x.device)
    for dy in range(-2, 3):
        rr = (2 * ar_y + dy).clamp(0, H - 1)
        for dx in range(-2, 3):
            cc = (2 * ar_x + dx).clamp(0, W - 1)
            out = out + BIN5[dy + 2] * BIN5[dx + 2] * x[rr][:, cc]
    return out


def _up_axis_torch(n, nc, device):
    c = (torch.arange(n, device=device, dtype=torch.float64) + 0.5) / 2 - 0.5
    i0 = torch.floor(c)
    f = c - i0
    i0 = i0.long()
    return i0.clamp(0, nc - 1), (i0 + 1).clamp(0, nc - 1), f


def upsample2_torch(c, H, W, scale=2.0):
    Hc, Wc = c.shape
    y0, y1, fy = _up_axis_torch(H, Hc, c.device)
    x0, x1, fx = _up_axis_torch(W, Wc, c.device)
    fy, fx = fy[:, None].to(c), fx[None, :].to(c)
    return scale * ((1 - fy) * ((1 - fx) * c[y0][:, x0] + fx * c[y0][:, x1])
                    + fy * ((1 - fx) * c[y1][:, x0] + fx * c[y1][:, x1]))


def warp_torch(src, ox, oy):
    """WarpImg2D rule; integer parts and the in-bounds test from the detached offsets."""
    H, W = src.shape
    mx = torch.floor(ox.detach()).long()
    my = torch.floor(oy.detach()).long()
    xf, yf = ox - mx.to(ox), oy - my.to(oy)
    Y, X = torch.meshgrid(torch.arange(H, device=src.device), torch.arange(W, device=src.device),
                          indexing="ij")
    ok = (X + mx >= 0) & (X + mx + 1 < W) & (Y + my >= 0) & (Y + my + 1 < H)
    bx = torch.where(ok, X + mx, torch.zeros_like(X))
    by = torch.where(ok, Y + my, torch.zeros_like(Y))
    bx1 = (bx + 1).clamp(max=W - 1)
    by1 = (by + 1).clamp(max=H - 1)
    o = (src[by, bx] * (1 - xf) * (1 - yf) + src[by, bx1] * xf * (1 - yf)
         + src[by1, bx] * (1 - xf) * yf + src[by1, bx1] * xf * yf)
    return torch.where(ok, o, src)


def coarse_to_fine_torch(I0, I1, alpha, levels, iters):
    p0, p1 = [I0], [I1]
    for _ in range(levels - 1):
        p0.append(blur_down_torch(p0[-1]))
        p1.append(blur_down_torch(p1[-1]))
    u = v = None
    for lev in range(levels - 1, -1, -1):
        if u is None:
            u, v = hs_torch(p0[lev], p1[lev], alpha, iters)
        else:
            H, W = p0[lev].shape
            uu, vv = upsample2_torch(u, H, W), upsample2_torch(v, H, W)
            du, dv = hs_torch(p0[lev], warp_torch(p1[lev], uu, vv), alpha, iters)
            u, v = uu + du, vv + dv
    return u, v
