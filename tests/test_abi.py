"""The C-ABI library: it loads, exports exactly what include/hsflow.h declares, and its
argument checks return the documented status before any device work (these calls
touch no GPU, so they run on CPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from hindemith_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^HS_API\s+[\w\s\*]*?\b(hs_\w+)\s*\(", src, flags=re.M)
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
        assert n in L.SIGNATURES, f"{n} has no ctypes signature in _lib.py"


def test_status_strings():
    for code in range(8):
        s = L.status_string(code)
        assert s and "unknown" not in s
    assert "unknown" in L.status_string(99)


def test_version():
    assert L.lib().hs_version() >= 100


def fake_ptr(offset=0):
    # never dereferenced: every call below fails its argument check first
    return ctypes.c_void_p(0x100000 + offset)


def test_argument_checks_before_launch():
    lib = L.lib()
    P = fake_ptr()
    w = np.ones(3, np.float32)
    o = np.zeros(3, np.int32)
    wp, op_ = w.ctypes.data_as(L._fp), o.ctypes.data_as(L._ip)
    # bad geometry
    assert lib.hs_stencil2d(wp, op_, op_, 3, P, fake_ptr(256), 0, 4, 4, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_stencil2d(wp, op_, op_, 3, P, fake_ptr(256), 4, 5, 4, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_stencil2d(wp, op_, op_, 3, P, fake_ptr(256), 4, 5, 6, None) == L.HS_ERR_ALIGNMENT
    # tap count
    assert lib.hs_stencil2d(wp, op_, op_, 0, P, fake_ptr(256), 4, 4, 4, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_stencil2d(wp, op_, op_, 65, P, fake_ptr(256), 4, 4, 4, None) == L.HS_ERR_INVALID_ARG
    # aliasing and alignment
    assert lib.hs_stencil2d(wp, op_, op_, 3, P, P, 4, 4, 4, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_stencil2d(wp, op_, op_, 3, fake_ptr(4), fake_ptr(256), 4, 4, 4, None) == L.HS_ERR_ALIGNMENT
    assert b"16-byte" in lib.hs_last_error()
    # bad op code
    assert lib.hs_array2d_op(7, P, P, P, 4, 4, 4, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_array2d_op(0, None, P, P, 4, 4, 4, None) == L.HS_ERR_INVALID_ARG


def test_sweep_argument_checks():
    lib = L.lib()
    P = fake_ptr()
    cfg = L.make_config()
    H, W, ld = 8, 8, 8
    need = lib.hs_sweeps_workspace_bytes(H, W, ld)
    assert need == 2 * 256  # two 8x8 float planes, each rounded to 256 bytes
    assert lib.hs_forward_workspace_bytes(H, W, ld) == 5 * 256
    # iters < 0
    st = lib.hs_sweeps(P, P, P, H, W, ld, 1.0, -1, P, P, P, need, ctypes.byref(cfg), None)
    assert st == L.HS_ERR_INVALID_ARG
    # iters == 0 is a no-op that needs no workspace
    st = lib.hs_sweeps(P, P, P, H, W, ld, 1.0, 0, P, P, None, 0, ctypes.byref(cfg), None)
    assert st == L.HS_OK
    # workspace too small
    st = lib.hs_sweeps(P, P, P, H, W, ld, 1.0, 5, P, P, P, need - 1, ctypes.byref(cfg), None)
    assert st == L.HS_ERR_WORKSPACE
    # T out of range, reserved fields
    bad = L.make_config(sweeps_per_pass=9)
    st = lib.hs_sweeps(P, P, P, H, W, ld, 1.0, 5, P, P, P, need, ctypes.byref(bad), None)
    assert st == L.HS_ERR_INVALID_ARG
    bad = L.make_config()
    bad.reserved[1] = 3
    st = lib.hs_forward(P, P, H, W, ld, 1.0, 5, P, P, P, 10 ** 6, ctypes.byref(bad), None)
    assert st == L.HS_ERR_INVALID_ARG
    # layout outside 0..2, and the 4-column layout without the fast form
    for bad in (L.make_config(layout=3), L.make_config(layout=2, fast_math=False)):
        st = lib.hs_forward(P, P, H, W, ld, 1.0, 5, P, P, P, 10 ** 6, ctypes.byref(bad), None)
        assert st == L.HS_ERR_INVALID_ARG
        assert "layout" in L.lib().hs_last_error().decode()
    st = lib.hs_forward(P, P, H, W, ld, 1.0, 5, P, P, P, 10, ctypes.byref(cfg), None)
    assert st == L.HS_ERR_WORKSPACE


def test_hs_error_raises_with_detail():
    with pytest.raises(L.HSError) as ei:
        L.check(L.lib().hs_array2d_op(9, fake_ptr(), fake_ptr(), fake_ptr(), 4, 4, 4, None), "hs_array2d_op")
    assert ei.value.status == L.HS_ERR_INVALID_ARG
    assert "op=9" in str(ei.value)


def test_batched_workspace_and_argument_checks():
    from hindemith_b200 import batched

    lib = L.lib()
    cfg = L.make_config(sweeps_per_pass=4)
    specs = [(240, 320, 1.0, 100), (7, 130, 0.5, 9)]
    nb = batched.workspace_bytes(specs, cfg)
    # header + 5 planes per pair + one counter per (segment, strip) tile
    planes = 5 * (240 * 320 * 4) + 5 * ((7 * 132 * 4 + 255) // 256 * 256)
    assert nb >= 256 + planes and nb % 256 == 0
    arr = (L.hs_pair_desc * 2)()
    for d, (H, W, a, n) in zip(arr, specs):
        d.H, d.W, d.ld, d.alpha, d.iters = H, W, (W + 3) // 4 * 4, a, n
    p = ctypes.c_void_p(0x100000)
    # n out of range, workspace too small, reserved != 0: rejected before device work
    assert lib.hs_forward_batched(arr, 0, p, nb, ctypes.byref(cfg), None, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_forward_batched(arr, 129, p, nb, ctypes.byref(cfg), None, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_forward_batched(arr, 2, p, nb - 1, ctypes.byref(cfg), None, None) == L.HS_ERR_WORKSPACE
    arr[1].reserved = 1
    assert lib.hs_forward_batched_workspace_bytes(arr, 2, ctypes.byref(cfg)) == 0
    assert lib.hs_forward_batched(arr, 2, p, nb, ctypes.byref(cfg), None, None) == L.HS_ERR_INVALID_ARG
    arr[1].reserved = 0
    arr[0].iters = -1
    assert lib.hs_forward_batched(arr, 2, p, nb, ctypes.byref(cfg), None, None) == L.HS_ERR_INVALID_ARG


def test_pyramid_argument_checks():
    lib = L.lib()
    P, Q = fake_ptr(), fake_ptr(256)
    # coarse stride below ceil(W/2), unaligned stride, null and unaligned planes, aliasing
    assert lib.hs_blur_down(P, 8, 8, 8, Q, 2, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_blur_down(P, 8, 6, 6, Q, 4, None) == L.HS_ERR_ALIGNMENT
    assert lib.hs_blur_down(None, 8, 8, 8, Q, 4, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_blur_down_adjoint(P, 0, 8, 8, 4, Q, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_upsample2(P, 2, Q, 8, 8, 8, 2.0, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_upsample2_adjoint(P, 8, 8, 8, fake_ptr(4), 4, 2.0, None) == L.HS_ERR_ALIGNMENT
    assert lib.hs_warp(P, P, P, 8, 8, 8, P, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_warp(P, P, None, 8, 8, 8, Q, None) == L.HS_ERR_INVALID_ARG
    need = lib.hs_warp_adjoint_workspace_bytes(8, 8, 8)
    assert need == 256 + 512
    assert lib.hs_warp_adjoint(P, P, P, P, 8, 7, 7, Q, Q, Q, Q, need, None) == L.HS_ERR_ALIGNMENT
    assert lib.hs_warp_adjoint(P, P, P, P, 8, 8, 8, Q, Q, Q, Q, need - 1, None) == L.HS_ERR_WORKSPACE
    assert lib.hs_warp_adjoint(P, P, P, P, 8, 8, 8, Q, Q, Q, None, need, None) == L.HS_ERR_WORKSPACE
    assert lib.hs_warp_adjoint(P, P, P, P, 8, 8, 8, Q, Q, Q, fake_ptr(16), need, None) == L.HS_ERR_ALIGNMENT


def test_epe_argument_checks_before_launch():
    lib = L.lib()
    P = fake_ptr()
    d = (L.hs_epe_pair * 2)()
    for x in d:
        x.u = x.v = x.ut = x.vt = 0x100000
        x.H, x.W, x.ld = 4, 4, 4
    assert lib.hs_epe_workspace_bytes(2) == 1024  # 2 x 64 doubles, rounded to 256
    assert lib.hs_epe_loss_batched(d, 0, 0.0, P, P, 1024, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_epe_loss_batched(d, 2, -1.0, P, P, 1024, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_epe_loss_batched(d, 2, 0.0, P, P, 512, None) == L.HS_ERR_WORKSPACE
    d[1].reserved = 1
    assert lib.hs_epe_loss_batched(d, 2, 0.0, P, P, 1024, None) == L.HS_ERR_INVALID_ARG
    d[1].reserved = 0
    d[1].ld = 6
    assert lib.hs_epe_loss_batched(d, 2, 0.0, P, P, 1024, None) == L.HS_ERR_ALIGNMENT
    d[1].ld = 4
    # the backward needs gradient planes
    assert lib.hs_epe_loss_backward_batched(d, 2, 0.0, P, None) == L.HS_ERR_INVALID_ARG


def test_cg_family_argument_checks():
    lib = L.lib()
    P = fake_ptr()
    cfg = L.make_config()
    assert lib.hs_matrix_powers(1.0, P, P, P, P, 8, 8, 8, 0, P, P, 64, ctypes.byref(cfg), None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_matrix_powers(1.0, P, P, P, P, 8, 8, 8, 3, P, P, 32, ctypes.byref(cfg), None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_matrix_powers(1.0, P, P, None, P, 8, 8, 8, 3, P, P, 64, ctypes.byref(cfg), None) == L.HS_ERR_INVALID_ARG
    deep = L.make_config(sweeps_per_pass=5)
    assert lib.hs_matrix_powers(1.0, P, P, P, P, 8, 8, 8, 3, P, P, 64, ctypes.byref(deep), None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_apply_hs_preconditioner(0.25, P, P, P, P, P, 8, 6, 6, P, P, None) == L.HS_ERR_ALIGNMENT
    assert lib.hs_apply_hs_preconditioner(0.25, P, P, P, P, P, 0, 8, 8, P, P, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_apply_hs_preconditioner(0.25, P, P, P, fake_ptr(8), P, 8, 8, 8, P, P, None) == L.HS_ERR_ALIGNMENT


def test_lk_brox_argument_checks():
    lib = L.lib()
    P = fake_ptr()
    assert lib.hs_lk_least_squares(P, P, P, 8, 8, 8, 0, P, P, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_lk_least_squares(P, P, P, 8, 8, 8, 17, P, P, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_lk_least_squares(P, None, P, 8, 8, 8, 2, P, P, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_set_brox_matrix(P, 8, 8, 8, 1.0, P, 32, 0, None, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_set_brox_matrix(P, 8, 8, 8, 1.0, P, 64, 1, None, None) == L.HS_ERR_INVALID_ARG
    ox = (ctypes.c_int * 17)()
    assert lib.hs_spmv_dia2d(P, 64, ox, ox, 17, P, 8, 8, 8, fake_ptr(256), None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_spmv_dia2d(P, 64, ox, ox, 5, P, 8, 8, 8, P, None) == L.HS_ERR_INVALID_ARG  # x == y
    assert lib.hs_apply_brox_preconditioner(P, P, P, P, P, P, 8, 8, 8, P, fake_ptr(2), None) == L.HS_ERR_ALIGNMENT


def test_selftest_wait_argument_checks():
    lib = L.lib()
    assert lib.hs_selftest_bounded_wait(None, 16, None) == L.HS_ERR_INVALID_ARG
    assert lib.hs_selftest_bounded_wait(fake_ptr(), 0, None) == L.HS_ERR_INVALID_ARG
