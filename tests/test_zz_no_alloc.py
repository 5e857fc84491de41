"""hs_forward_noalloc: the plain forward for callers that cannot allocate device memory
(a frame loop that must not call cudaMalloc/cudaFree, which can synchronise the
device, or a host binding that cannot own a device buffer).  Its scratch is a static
array inside libhsflow, so the test checks that it gives hs_forward's results, call
after call, and that it refuses sizes its scratch cannot hold.

This file sorts last so that a run stopping at the first failure has already run every
other test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from hindemith_b200 import _lib as L


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    # rejected by the size check, before any device work: runs without a GPU too
    lib = L.lib()
    H, W = 2048, 2048  # five 16 MiB planes > 48 MiB
    p = ctypes.c_void_p(0x100000)
    cfg = L.make_config()
    st = lib.hs_forward_noalloc(p, p, H, W, W, 1.0, 10, p, p, ctypes.byref(cfg), None)
    assert st == L.HS_ERR_WORKSPACE
    assert b"static scratch" in lib.hs_last_error()
    assert lib.hs_forward_workspace_bytes(H, W, W) > L.HS_NOALLOC_SCRATCH_BYTES


def test_noalloc_size_limit_is_exact():
    """Planes of exactly HS_NOALLOC_SCRATCH_BYTES / 5 rounded down to 256 bytes (2313 rows of
    ld 1088: 10,066,176 bytes) pass the size check; one more row is rejected.  The pointers
    are misaligned on purpose, so a call past the size check stops at the argument checks
    (or, without a GPU, at the device lookup) and no kernel ever runs."""
    lib = L.lib()
    W = ld = 1088
    assert 2313 * ld * 4 == 10066176 == L.HS_NOALLOC_SCRATCH_BYTES // 5 // 256 * 256
    bad = ctypes.c_void_p(0x100004)  # 4-byte aligned, not 16: HS_ERR_ALIGNMENT after the size check
    cfg = L.make_config()
    st = lib.hs_forward_noalloc(bad, bad, 2313, W, ld, 1.0, 10, bad, bad, ctypes.byref(cfg), None)
    assert st != L.HS_ERR_WORKSPACE, lib.hs_last_error()
    assert st in (L.HS_ERR_ALIGNMENT, L.HS_ERR_CUDA, L.HS_ERR_NO_DEVICE), st
    st = lib.hs_forward_noalloc(bad, bad, 2314, W, ld, 1.0, 10, bad, bad, ctypes.byref(cfg), None)
    assert st == L.HS_ERR_WORKSPACE


@pytest.mark.gpu
@pytest.mark.parametrize("fast", [False, True])
def test_noalloc_matches_hs_forward_twice(fast):
    import torch

    from hindemith_b200 import device as D
    from hindemith_b200 import synthetic

    assert torch.cuda.is_available(), "gpu test without a CUDA device"
    lib = L.lib()
    H, W = 300, 518  # W not a multiple of 4: padded rows (ld = 520)
    cfg = L.make_config(sweeps_per_pass=4, fast_math=fast)
    outs = []
    for seed in (1000, 1001):  # two calls in a row, different inputs
        I0h, I1h, _, _ = synthetic.make_pair(H, W, seed=seed)
        I0 = D.as_plane(torch.from_numpy(I0h).cuda())
        I1 = D.as_plane(torch.from_numpy(I1h).cuda())
        ld = D.ld_of(I0)
        ref_u, ref_v = D.hs_forward(I0, I1, 0.8, 37, cfg)
        uv = D.empty_planes(2, H, W)
        u, v = uv[0], uv[1]
        u.fill_(123.0), v.fill_(-7.0)  # stale output contents must not leak in
        st = lib.hs_forward_noalloc(D.ptr(I0), D.ptr(I1), H, W, ld, 0.8, 37, D.ptr(u), D.ptr(v),
                                    ctypes.byref(cfg), D.stream_handle())
        L.check(st, "hs_forward_noalloc")
        torch.cuda.synchronize()
        assert np.array_equal(_bits(u.cpu().numpy()), _bits(ref_u.cpu().numpy()))
        assert np.array_equal(_bits(v.cpu().numpy()), _bits(ref_v.cpu().numpy()))
        outs.append(u.cpu().numpy())
    assert not np.array_equal(outs[0], outs[1])  # the second call did its own work


@pytest.mark.gpu
def test_noalloc_full_hd_matches_hs_forward():
    """The size the scratch is dimensioned for, 1920x1080, bit for bit against hs_forward,
    two calls in a row."""
    import torch

    from hindemith_b200 import device as D
    from hindemith_b200 import synthetic

    assert torch.cuda.is_available(), "gpu test without a CUDA device"
    lib = L.lib()
    H, W = 1080, 1920
    cfg = L.make_config(fast_math=True)
    for seed in (1000, 1001):
        I0h, I1h, _, _ = synthetic.make_pair(H, W, seed=seed)
        I0 = D.as_plane(torch.from_numpy(I0h).cuda())
        I1 = D.as_plane(torch.from_numpy(I1h).cuda())
        ref_u, ref_v = D.hs_forward(I0, I1, 1.0, 50, cfg)
        uv = D.empty_planes(2, H, W)
        st = lib.hs_forward_noalloc(D.ptr(I0), D.ptr(I1), H, W, D.ld_of(I0), 1.0, 50,
                                    D.ptr(uv[0]), D.ptr(uv[1]), ctypes.byref(cfg),
                                    D.stream_handle())
        L.check(st, "hs_forward_noalloc")
        torch.cuda.synchronize()
        assert np.array_equal(_bits(uv[0].cpu().numpy()), _bits(ref_u.cpu().numpy()))
        assert np.array_equal(_bits(uv[1].cpu().numpy()), _bits(ref_v.cpu().numpy()))
