"""Parity of the CUDA path (through the C ABI) with the oracle and the golden fixtures.

Tolerances: exact mode (the default) must be bit-identical to the reference's FP32
semantics; fast mode must stay within 1e-4 max-abs of the exact result and of the
FP64 oracle."""
import numpy as np
import pytest
import torch

from conftest import assert_bitexact, golden, golden_files
from hindemith_b200 import _lib as L
from hindemith_b200 import device as D
from hindemith_b200 import synthetic
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-4
# Every depth the library accepts (and the autotuner may pick): 1 .. HS_MAX_SWEEPS_PER_PASS.
ALL_T = list(range(1, L.HS_MAX_SWEEPS_PER_PASS + 1))


def dev(a, pad=0):
    """numpy (H, W) -> plane on the GPU; `pad` extra floats of row padding."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    H, W = a.shape
    ld = D.padded_ld(W) + 4 * pad
    buf = torch.zeros((H, ld), dtype=torch.float32, device="cuda")
    buf[:, :W] = torch.from_numpy(a).cuda()
    return buf[:, :W]


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("path", golden_files("stencil_*.npz"))
@pytest.mark.parametrize("pad", [0, 3])
def test_stencil2d_golden(cuda, path, pad):
    d = np.load(path)
    for i, _ in enumerate(d["shapes"]):
        x, ref = d[f"x{i}"], d[f"out{i}"]
        out = D.stencil2d(d["weights"], d["offx"], d["offy"], dev(x, pad))
        assert_bitexact(host(out), ref, f"{path} {i}")


@pytest.mark.parametrize("pad", [0, 3])
def test_stencil2d_against_reference_template_golden(cuda, pad):
    """Stencil2DMVM's device template run as C (clamped taps, accumulation from 0 in tap
    order), including an asymmetric 6-tap stencil with offsets up to 5: bit-identical."""
    g = golden("tmpl_stencil.npz")
    for i in range(int(g["n"])):
        out = D.stencil2d(g[f"w_{i}"], g[f"offx_{i}"], g[f"offy_{i}"], dev(g[f"x_{i}"], pad))
        assert_bitexact(host(out), g[f"out_{i}"], f"case {i}")


def test_pointwise_ops(cuda):
    rng = np.random.default_rng(1)
    b = rng.standard_normal((37, 45)).astype(np.float32)
    c = rng.standard_normal((37, 45)).astype(np.float32)
    s = np.float32(0.731)
    for op, f in ((L.HS_OP_ADD, np.add), (L.HS_OP_SUB, np.subtract), (L.HS_OP_MUL, np.multiply),
                  (L.HS_OP_DIV, np.divide)):
        assert_bitexact(host(D.array2d_op(op, dev(b), dev(c))), f(b, c), f"op {op}")
        assert_bitexact(host(D.array2d_scalar_op(op, dev(b), s)), f(b, s), f"scalar op {op}")
        assert_bitexact(host(D.scalar_array2d_op(op, s, dev(b))), f(s, b), f"op scalar {op}")
    assert_bitexact(host(D.array2d_copy(dev(b))), b, "copy")


@pytest.mark.parametrize("path", golden_files("hs_*.npz"))
def test_derivs_golden(cuda, path):
    d = np.load(path)
    Ix, Iy, It = D.hs_derivs(dev(d["I0"]), dev(d["I1"]))
    for t, name in ((Ix, "Ix"), (Iy, "Iy"), (It, "It")):
        assert_bitexact(host(t), d[name], name)


def run_sweeps(Ix, Iy, It, alpha2, iters, u0, v0, **cfg):
    Ixd, Iyd, Itd = (dev(a) for a in (Ix, Iy, It))
    u, v = dev(u0), dev(v0)
    D.hs_sweeps(Ixd, Iyd, Itd, alpha2, iters, u, v, L.make_config(**cfg))
    return host(u), host(v)


@pytest.mark.parametrize("path", golden_files("hs_*.npz"))
@pytest.mark.parametrize("T", ALL_T)
def test_sweeps_exact_golden(cuda, path, T):
    d = np.load(path)
    z = np.zeros_like(d["I0"])
    for seg in (0, 1, 3):
        u, v = run_sweeps(d["Ix"], d["Iy"], d["It"], d["alpha2"], int(d["sweeps"]), z, z,
                          sweeps_per_pass=T, rows_per_segment=seg)
        assert_bitexact(u, d["u"], f"u T={T} seg={seg}")
        assert_bitexact(v, d["v"], f"v T={T} seg={seg}")


@pytest.mark.parametrize("shape", [(1, 1), (1, 2), (1, 67), (67, 1), (2, 2), (3, 5), (5, 3),
                                   (7, 130), (130, 7), (64, 64), (65, 127), (50, 4), (33, 500),
                                   (97, 256)])
@pytest.mark.parametrize("T", ALL_T)
def test_sweeps_exact_edge_shapes(cuda, shape, T):
    H, W = shape
    rng = np.random.default_rng(H * 1000 + W)
    Ix, Iy, It = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(3))
    u0, v0 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(2))
    iters = 2 * T + 1  # a partial last pass
    ru, rv = O.hs_sweeps(Ix, Iy, It, np.float32(0.8), iters, u0, v0)
    u, v = run_sweeps(Ix, Iy, It, np.float32(0.8), iters, u0, v0, sweeps_per_pass=T)
    assert_bitexact(u, ru, "u")
    assert_bitexact(v, rv, "v")


@pytest.mark.parametrize("iters", [0, 1, 3, 4, 5, 9, 16])
def test_sweeps_pass_parity(cuda, iters):
    """Even and odd pass counts, partial passes and iters = 0 all end in (u, v)."""
    d = golden("hs_24x31.npz")
    rng = np.random.default_rng(iters)
    u0, v0 = (rng.standard_normal(d["I0"].shape).astype(np.float32) for _ in range(2))
    ru, rv = O.hs_sweeps(d["Ix"], d["Iy"], d["It"], d["alpha2"], iters, u0, v0)
    u, v = run_sweeps(d["Ix"], d["Iy"], d["It"], d["alpha2"], iters, u0, v0, sweeps_per_pass=4)
    assert_bitexact(u, ru, "u")
    assert_bitexact(v, rv, "v")


@pytest.mark.parametrize("T", ALL_T)
@pytest.mark.parametrize("layout", [1, 2])
def test_sweeps_fast_within_tolerance(cuda, T, layout):
    """The fast form at every depth, in both layouts (2 and 4 columns per lane), stays
    within 1e-4 max-abs of the FP64 oracle."""
    I0, I1, _, _ = synthetic.make_pair(160, 200, seed=1003)
    Ix, Iy, It = O.c_hs_derivs(I0, I1)
    z = np.zeros_like(I0)
    u64, v64 = O.c_hs_sweeps(Ix, Iy, It, 1.0, 200, z, z, np.float64)
    u, v = run_sweeps(Ix, Iy, It, 1.0, 200, z, z, sweeps_per_pass=T, fast_math=True,
                      layout=layout)
    assert np.abs(u - u64).max() < FAST_TOL
    assert np.abs(v - v64).max() < FAST_TOL


def test_forward_config0_shape(cuda):
    """256x256, 100 sweeps, alpha 1: bit-identical to the oracle, and its distance to the
    FP64 oracle is the reference's own FP32 error."""
    I0, I1, _, _ = synthetic.generate(synthetic.plain_256())
    ru, rv = O.c_hs_forward(I0, I1, 1.0, 100)
    u64, v64 = O.c_hs_forward(I0, I1, 1.0, 100, np.float64)
    for T in (1, 4):
        u, v = D.hs_forward(dev(I0), dev(I1), 1.0, 100, L.make_config(sweeps_per_pass=T))
        assert_bitexact(host(u), ru, "u")
        assert_bitexact(host(v), rv, "v")
    assert np.abs(ru - u64).max() < 1e-5 and np.abs(rv - v64).max() < 1e-5
    uf, vf = D.hs_forward(dev(I0), dev(I1), 1.0, 100, L.make_config(fast_math=True))
    assert np.abs(host(uf) - u64).max() < FAST_TOL and np.abs(host(vf) - v64).max() < FAST_TOL


def test_forward_full_size_1080p(cuda):
    """1920x1080, 500 sweeps: the temporally blocked exact kernel equals the one-sweep
    kernel bit for bit (a size-independent property); 100 sweeps equal the C oracle;
    the fast form stays within 1e-4 of the exact one."""
    I0, I1, _, _ = synthetic.generate(synthetic.plain_1080p())
    a, b = dev(I0), dev(I1)
    u1, v1 = (host(t) for t in D.hs_forward(a, b, 1.0, 500, L.make_config(sweeps_per_pass=1)))
    u4, v4 = (host(t) for t in D.hs_forward(a, b, 1.0, 500, L.make_config(sweeps_per_pass=4)))
    assert_bitexact(u4, u1, "u")
    assert_bitexact(v4, v1, "v")
    uf, vf = (host(t) for t in D.hs_forward(a, b, 1.0, 500, L.make_config(fast_math=True)))
    assert np.abs(uf - u1).max() < FAST_TOL and np.abs(vf - v1).max() < FAST_TOL
    ru, rv = O.c_hs_forward(I0, I1, 1.0, 100)
    u, v = (host(t) for t in D.hs_forward(a, b, 1.0, 100))
    assert_bitexact(u, ru, "u@100")
    assert_bitexact(v, rv, "v@100")


def test_nondefault_stream_and_padding(cuda):
    d = golden("hs_70x130.npz")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        Ix, Iy, It = (dev(d[k], pad=2) for k in ("Ix", "Iy", "It"))
        u, v = dev(np.zeros_like(d["I0"]), pad=2), dev(np.zeros_like(d["I0"]), pad=2)
        D.hs_sweeps(Ix, Iy, It, d["alpha2"], int(d["sweeps"]), u, v, stream=s)
    s.synchronize()
    assert_bitexact(u.cpu().numpy(), d["u"], "u")
    assert_bitexact(v.cpu().numpy(), d["v"], "v")


def test_side_stream_with_growing_sizes(cuda):
    """hs_forward on a side stream, the size growing call by call (so the cached scratch is
    replaced each time), while the current stream allocates and overwrites memory: every
    flow equals the same call on the current stream, bit for bit."""
    s = torch.cuda.Stream()
    keep, refs, outs = [], [], []
    for i, (H, W) in enumerate([(64, 96), (200, 300), (400, 610), (700, 1030)]):
        I0, I1, _, _ = synthetic.make_pair(H, W, seed=700 + i)
        a, b = dev(I0), dev(I1)
        keep.append((a, b))
        refs.append(tuple(host(t) for t in D.hs_forward(a, b, 1.0, 40)))
        s.wait_stream(torch.cuda.current_stream())
        outs.append(D.hs_forward(a, b, 1.0, 40, stream=s))
        junk = torch.full((4 * H * W,), float("nan"), device="cuda")  # reuses freed memory
        del junk
    torch.cuda.synchronize()
    for (u, v), (ru, rv) in zip(outs, refs):
        assert_bitexact(u.cpu().numpy(), ru, "u")
        assert_bitexact(v.cpu().numpy(), rv, "v")


def test_misaligned_plane_is_rejected(cuda):
    base = torch.zeros((8, 12), device="cuda")
    shifted = base.view(-1)[1:1 + 8 * 8].view(8, 8)  # starts 4 bytes into the buffer
    lib = L.lib()
    st = lib.hs_array2d_copy(D.ptr(shifted), D.ptr(base), 8, 8, 8, None)
    assert st == L.HS_ERR_ALIGNMENT


WIDE_SHAPES = [(1, 1), (1, 5), (67, 1), (1, 67), (3, 5), (2, 200), (130, 257), (257, 130), (64, 128),
               (97, 256), (33, 500), (50, 4)]  # W % 4 == 0: the side strips' 2-select clamp


@pytest.mark.parametrize("shape", WIDE_SHAPES)
@pytest.mark.parametrize("T", ALL_T)
def test_wide_layout_equals_narrow(cuda, shape, T):
    """The fast form's 4-columns-per-lane layout computes every cell with the same
    arithmetic as the 2-column one: identical results, bit for bit, at every shape, depth
    and segmentation."""
    H, W = shape
    rng = np.random.default_rng(H * 1000 + W + T)
    Ix, Iy, It, u0, v0 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(5))
    ref = run_sweeps(Ix, Iy, It, 0.8, 23, u0, v0, sweeps_per_pass=T, fast_math=True, layout=1)
    for seg in (0, 3):
        got = run_sweeps(Ix, Iy, It, 0.8, 23, u0, v0, sweeps_per_pass=T, fast_math=True,
                         layout=2, rows_per_segment=seg)
        assert_bitexact(got[0], ref[0], "u")
        assert_bitexact(got[1], ref[1], "v")


@pytest.mark.parametrize("shape", [(1544, 2040), (1543, 2043)])
@pytest.mark.parametrize("T", ALL_T)
def test_wide_layout_equals_narrow_large(cuda, shape, T):
    """From 3 Mpx up the wide kernel runs its main loop unrolled two steps, a separate
    instantiation from the rolled loop of the smaller shapes above: bit-identical to the
    2-column layout there too (W % 4 == 0 and not)."""
    H, W = shape
    assert H * W >= 3000000
    rng = np.random.default_rng(H + W + T)
    Ix, Iy, It, u0, v0 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(5))
    ref = run_sweeps(Ix, Iy, It, 0.8, 23, u0, v0, sweeps_per_pass=T, fast_math=True, layout=1)
    got = run_sweeps(Ix, Iy, It, 0.8, 23, u0, v0, sweeps_per_pass=T, fast_math=True, layout=2)
    assert_bitexact(got[0], ref[0], "u")
    assert_bitexact(got[1], ref[1], "v")


@pytest.mark.parametrize("T", ALL_T)
def test_exact_form_large_equals_the_oracle(cuda, T):
    """A large image (3.15 Mpx) in the exact form, at every depth (the 2-column kernel's main
    loop rolled from depth 3, unrolled two steps below): equal to the FP32 C oracle bit for
    bit."""
    H, W = 1543, 2043
    rng = np.random.default_rng(7 + T)
    Ix, Iy, It, u0, v0 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(5))
    got = run_sweeps(Ix, Iy, It, 0.8, 2 * T + 1, u0, v0, sweeps_per_pass=T, fast_math=False)
    ru, rv = O.c_hs_sweeps(Ix, Iy, It, 0.8, 2 * T + 1, u0, v0)
    assert_bitexact(got[0], ru, "u")
    assert_bitexact(got[1], rv, "v")


def test_wide_layout_full_size(cuda):
    """1920x1080, 60 sweeps: the automatic layout (wide at this size) equals the narrow one
    and stays within 1e-4 of FP64."""
    I0, I1, _, _ = synthetic.generate(synthetic.plain_1080p())
    Ix, Iy, It = O.c_hs_derivs(I0, I1)
    z = np.zeros_like(I0)
    ref = run_sweeps(Ix, Iy, It, 1.0, 60, z, z, sweeps_per_pass=5, fast_math=True, layout=1)
    got = run_sweeps(Ix, Iy, It, 1.0, 60, z, z, sweeps_per_pass=5, fast_math=True, layout=0)
    assert_bitexact(got[0], ref[0], "u")
    assert_bitexact(got[1], ref[1], "v")
    u64, v64 = O.c_hs_sweeps(Ix, Iy, It, 1.0, 60, z, z, np.float64)
    assert np.abs(got[0] - u64).max() < FAST_TOL and np.abs(got[1] - v64).max() < FAST_TOL


def test_autotuner_candidates_are_all_pinned():
    """Every depth the autotuners may pick is one the parity tests above run."""
    from hindemith_b200 import autotune

    assert set(autotune.T_CANDIDATES) <= set(ALL_T)
    assert {c[0] for c in autotune.BATCH_CANDIDATES} <= set(ALL_T)


@pytest.mark.parametrize("fast", [True, False])
def test_plain_1080p_500_at_the_tuned_config(cuda, fast):
    """The headline workload exactly as the benchmark runs it: 1920x1080, 500 sweeps,
    alpha 1, at the (depth, segment, layout) the autotuner picks on this device.  The fast
    form stays within 1e-4 max-abs of the FP64 oracle; the exact form equals the FP32 C
    oracle bit for bit."""
    from hindemith_b200 import autotune

    spec = synthetic.plain_1080p()
    I0, I1, _, _ = synthetic.generate(spec)
    a, b = dev(I0), dev(I1)
    T, seg, layout = autotune.best_sweep_config(spec.H, spec.W, D.ld_of(a), fast_math=fast,
                                                sweeps=spec.iters)
    cfg = L.make_config(sweeps_per_pass=T, rows_per_segment=seg, fast_math=fast, layout=layout)
    u, v = (host(t) for t in D.hs_forward(a, b, spec.alpha, spec.iters, cfg))
    if fast:
        u64, v64 = O.c_hs_forward(I0, I1, spec.alpha, spec.iters, np.float64)
        eu, ev = np.abs(u - u64).max(), np.abs(v - v64).max()
        assert eu < FAST_TOL and ev < FAST_TOL, (T, seg, layout, eu, ev)
    else:
        ru, rv = O.c_hs_forward(I0, I1, spec.alpha, spec.iters)
        assert_bitexact(u, ru, f"u T={T} seg={seg}")
        assert_bitexact(v, rv, f"v T={T} seg={seg}")
