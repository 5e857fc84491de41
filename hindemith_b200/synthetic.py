"""Seeded synthetic Horn-Schunck inputs (the benchmark workloads' stand-in data).

No public dataset backs the reference's path, so image pairs are generated:

* I0: uniform [0, 1) noise from NumPy's PCG64 (seed 1000 + pair index), Gaussian blur
  of `sigma` px (reflect boundary), min-max renormalised to [0, 1].
* Ground-truth flow (u*, v*): per component, sum of three sinusoids
  a_k sin(2 pi (cos th_k x + sin th_k y) / lam_k + phi_k) with lam_k ~ U[32, 128] px,
  th_k, phi_k ~ U[0, 2 pi), a_k ~ U[0.5, 1]; each component is then scaled so that its
  maximum absolute value is `amplitude` px.
* I1(x) = I0(x - w(x)), bilinear with clamped coordinates, plus N(0, noise_std) noise
  (noise_std = 0.01, read as a standard deviation).

All outputs are float32, shape (H, W).  Draw order from the pair's generator: I0 noise,
flow parameters (u then v), I1 noise.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np


def _flow_component(rng, H, W, amplitude):
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    w = np.zeros((H, W), dtype=np.float64)
    for _ in range(3):
        lam = rng.uniform(32.0, 128.0)
        th = rng.uniform(0.0, 2 * np.pi)
        phi = rng.uniform(0.0, 2 * np.pi)
        a = rng.uniform(0.5, 1.0)
        w += a * np.sin(2 * np.pi * (np.cos(th) * x + np.sin(th) * y) / lam + phi)
    m = np.abs(w).max()
    if m > 0:
        w *= amplitude / m
    return w


def bilinear_clamped(img: np.ndarray, xs: np.ndarray, ys: np.ndarray) -> np.ndarray:
    H, W = img.shape
    xs = np.clip(xs, 0.0, W - 1.0)
    ys = np.clip(ys, 0.0, H - 1.0)
    x0 = np.floor(xs).astype(np.int64)
    y0 = np.floor(ys).astype(np.int64)
    x1 = np.minimum(x0 + 1, W - 1)
    y1 = np.minimum(y0 + 1, H - 1)
    fx = xs - x0
    fy = ys - y0
    im = img.astype(np.float64)
    return ((1 - fx) * (1 - fy) * im[y0, x0] + fx * (1 - fy) * im[y0, x1]
            + (1 - fx) * fy * im[y1, x0] + fx * fy * im[y1, x1])


def make_pair(H: int, W: int, seed: int, sigma: float = 2.0, amplitude: float = 1.5,
              noise_std: float = 0.01):
    """(I0, I1, u_true, v_true), float32 (H, W)."""
    from scipy.ndimage import gaussian_filter

    rng = np.random.Generator(np.random.PCG64(seed))
    I0 = rng.random((H, W))
    I0 = gaussian_filter(I0, sigma=sigma, mode="reflect")
    lo, hi = I0.min(), I0.max()
    I0 = (I0 - lo) / (hi - lo) if hi > lo else np.zeros_like(I0)
    u = _flow_component(rng, H, W, amplitude)
    v = _flow_component(rng, H, W, amplitude)
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    I1 = bilinear_clamped(I0, x - u, y - v) + rng.normal(0.0, noise_std, size=(H, W))
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return f32(I0), f32(I1), f32(u), f32(v)


# ------------------------------------------------------------------ workloads

@dataclass
class PairSpec:
    index: int
    H: int
    W: int
    alpha: float
    iters: int
    seed: int
    sigma: float = 2.0
    amplitude: float = 1.5


BATCH_RESOLUTIONS = [(240, 320), (480, 640), (720, 1280), (1080, 1920), (2048, 2048)]
BATCH_ITERS = [100, 200, 500]


def plain_1080p() -> PairSpec:
    """One 1920x1080 pair, blur 3 px, flow up to 2 px, alpha 1, 500 sweeps."""
    return PairSpec(0, 1080, 1920, 1.0, 500, 1000, sigma=3.0, amplitude=2.0)


def plain_256() -> PairSpec:
    """One 256x256 pair, blur 2 px, flow up to 1.5 px, alpha 1, 100 sweeps (CPU parity)."""
    return PairSpec(0, 256, 256, 1.0, 100, 1000, sigma=2.0, amplitude=1.5)


def batch_mixed(n: int = 64, seed: int = 2024) -> List[PairSpec]:
    """n pairs with resolution, alpha and sweep count drawn per pair (seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        H, W = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
        alpha = float(np.float32(rng.uniform(0.5, 2.0)))
        iters = BATCH_ITERS[int(rng.integers(len(BATCH_ITERS)))]
        out.append(PairSpec(i, H, W, alpha, iters, 1000 + i))
    return out


def batch_512(n: int = 16) -> List[PairSpec]:
    """n 512x512 pairs, alpha 1, 200 sweeps (the differentiable workload)."""
    return [PairSpec(i, 512, 512, 1.0, 200, 1000 + i) for i in range(n)]


def batch_pyramid(n: int = 8) -> List[PairSpec]:
    """n 2048x2048 pairs with large flow (up to 12 px), alpha 1, 100 sweeps per level (the
    coarse-to-fine workload)."""
    return [PairSpec(i, 2048, 2048, 1.0, 100, 3000 + i, sigma=2.0, amplitude=12.0) for i in range(n)]


def generate(spec: PairSpec):
    return make_pair(spec.H, spec.W, spec.seed, spec.sigma, spec.amplitude)
