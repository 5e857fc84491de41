"""ctypes binding of libhsflow.so (the C ABI declared in include/hsflow.h).

The library is the only compute path of this package: importing a compute entry point
without a built library raises immediately; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libhsflow.so")

HS_OK = 0
HS_ERR_INVALID_ARG = 1
HS_ERR_ALIGNMENT = 2
HS_ERR_WORKSPACE = 3
HS_ERR_CUDA = 4
HS_ERR_TIMEOUT = 5
HS_ERR_UNSUPPORTED = 6
HS_ERR_NO_DEVICE = 7

HS_OP_ADD, HS_OP_SUB, HS_OP_MUL, HS_OP_DIV = 0, 1, 2, 3
HS_MAX_TAPS = 64
HS_MAX_SWEEPS_PER_PASS = 8

# Python AST operator class name -> hs_binop, the names the reference's templates
# carry in their 'op' property (Templates.py:112, Array2DOp.cpp:36-51).
OP_CODES = {"Add": HS_OP_ADD, "Sub": HS_OP_SUB, "Mult": HS_OP_MUL, "Div": HS_OP_DIV}


class HSError(RuntimeError):
    """A libhsflow call returned a status other than HS_OK."""

    def __init__(self, status: int, func: str, detail: str):
        self.status = status
        self.func = func
        self.detail = detail
        super().__init__(f"{func}: {status_string(status)} ({detail})")


class hs_config(ctypes.Structure):
    _fields_ = [
        ("sweeps_per_pass", ctypes.c_int),
        ("rows_per_segment", ctypes.c_int),
        ("fast_math", ctypes.c_int),
        ("avg_edge", ctypes.c_float),
        ("avg_corner", ctypes.c_float),
        ("layout", ctypes.c_int), ("reserved", ctypes.c_int * 2),
    ]


class hs_pair_desc(ctypes.Structure):
    _fields_ = [("I0", ctypes.c_void_p), ("I1", ctypes.c_void_p), ("u", ctypes.c_void_p),
                ("v", ctypes.c_void_p), ("H", ctypes.c_int), ("W", ctypes.c_int),
                ("ld", ctypes.c_int), ("alpha", ctypes.c_float), ("iters", ctypes.c_int),
                ("reserved", ctypes.c_int)]


HS_MAX_BATCH = 128


HS_FUSED_MAX_IN, HS_FUSED_MAX_OUT, HS_FUSED_MAX_SCALARS, HS_FUSED_MAX_SUMS = 16, 8, 64, 8


class hs_fused_args(ctypes.Structure):
    _fields_ = [("in_", ctypes.c_void_p * HS_FUSED_MAX_IN), ("out", ctypes.c_void_p * HS_FUSED_MAX_OUT),
                ("s", ctypes.c_float * HS_FUSED_MAX_SCALARS), ("H", ctypes.c_int),
                ("W", ctypes.c_int), ("ld", ctypes.c_int), ("nsums", ctypes.c_int),
                ("sums", ctypes.c_void_p), ("reserved", ctypes.c_int * 4)]


class hs_epe_pair(ctypes.Structure):
    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("ut", ctypes.c_void_p),
                ("vt", ctypes.c_void_p), ("du", ctypes.c_void_p), ("dv", ctypes.c_void_p),
                ("H", ctypes.c_int), ("W", ctypes.c_int), ("ld", ctypes.c_int),
                ("reserved", ctypes.c_int)]


class hs_train_pair(ctypes.Structure):
    _fields_ = [("I0", ctypes.c_void_p), ("I1", ctypes.c_void_p), ("u", ctypes.c_void_p),
                ("v", ctypes.c_void_p), ("alpha", ctypes.c_void_p), ("dLdu", ctypes.c_void_p),
                ("dLdv", ctypes.c_void_p), ("dI0", ctypes.c_void_p), ("dI1", ctypes.c_void_p),
                ("dalpha", ctypes.c_void_p), ("H", ctypes.c_int), ("W", ctypes.c_int),
                ("ld", ctypes.c_int), ("reserved", ctypes.c_int)]


HS_MAX_TRAIN_PAIRS = 32

_lib = None
_lock = threading.Lock()

_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_sz = ctypes.c_size_t
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)
_cfgp = ctypes.POINTER(hs_config)
_pdp = ctypes.POINTER(hs_pair_desc)
_tpp = ctypes.POINTER(hs_train_pair)
_epp = ctypes.POINTER(hs_epe_pair)

# name -> (restype, argtypes)
SIGNATURES = {
    "hs_status_string": (ctypes.c_char_p, [_i]),
    "hs_last_error": (ctypes.c_char_p, []),
    "hs_version": (_i, []),
    "hs_stencil2d": (_i, [_fp, _ip, _ip, _i, _vp, _vp, _i, _i, _i, _vp]),
    "hs_array2d_op": (_i, [_i, _vp, _vp, _vp, _i, _i, _i, _vp]),
    "hs_array2d_scalar_op": (_i, [_i, _vp, _f, _vp, _i, _i, _i, _vp]),
    "hs_scalar_array2d_op": (_i, [_i, _f, _vp, _vp, _i, _i, _i, _vp]),
    "hs_array2d_copy": (_i, [_vp, _vp, _i, _i, _i, _vp]),
    "hs_derivs": (_i, [_vp, _vp, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "hs_sweeps_workspace_bytes": (_sz, [_i, _i, _i]),
    "hs_sweeps": (_i, [_vp, _vp, _vp, _i, _i, _i, _f, _i, _vp, _vp, _vp, _sz, _cfgp, _vp]),
    "hs_forward_workspace_bytes": (_sz, [_i, _i, _i]),
    "hs_forward": (_i, [_vp, _vp, _i, _i, _i, _f, _i, _vp, _vp, _vp, _sz, _cfgp, _vp]),
    "hs_forward_noalloc": (_i, [_vp, _vp, _i, _i, _i, _f, _i, _vp, _vp, _cfgp, _vp]),
    "hs_forward_batched_workspace_bytes": (_sz, [_pdp, _i, _cfgp]),
    "hs_forward_batched": (_i, [_pdp, _i, _vp, _sz, _cfgp, _vp, _vp]),
    "hs_derivs_bytes": (_sz, [_i, _i, _i]),
    "hs_checkpoint_bytes": (_sz, [_i, _i, _i, _i, _i]),
    "hs_forward_train_workspace_bytes": (_sz, [_i, _i, _i]),
    "hs_forward_train": (_i, [_vp, _vp, _i, _i, _i, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _sz,
                              _cfgp, _vp]),
    "hs_backward_workspace_bytes": (_sz, [_i, _i, _i, _i]),
    "hs_train_workspace_bytes": (_sz, [_tpp, _i, _i, _i]),
    "hs_forward_train_batched": (_i, [_tpp, _i, _i, _i, _vp, _sz, _cfgp, _vp]),
    "hs_backward_batched": (_i, [_tpp, _i, _i, _i, _vp, _sz, _cfgp, _vp]),
    "hs_matrix_powers": (_i, [_f, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _sz, _cfgp, _vp]),
    "hs_apply_hs_preconditioner": (_i, [_f, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp]),
    "hs_selftest_bounded_wait": (_i, [_vp, _i, _vp]),
    "hs_lk_least_squares": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp]),
    "hs_set_brox_matrix": (_i, [_vp, _i, _i, _i, _f, _vp, _sz, _i, _vp, _vp]),
    "hs_spmv_dia2d": (_i, [_vp, _sz, _ip, _ip, _i, _vp, _i, _i, _i, _vp, _vp]),
    "hs_apply_brox_preconditioner": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp]),
    "hs_fused_workspace_bytes": (_sz, [_i, _i, _i]),
    "hs_fused_launch": (_i, [ctypes.c_char_p, _i, ctypes.POINTER(hs_fused_args), _vp, _sz, _vp]),
    "hs_epe_workspace_bytes": (_sz, [_i]),
    "hs_epe_loss_batched": (_i, [_epp, _i, _f, _vp, _vp, _sz, _vp]),
    "hs_epe_loss_backward_batched": (_i, [_epp, _i, _f, _vp, _vp]),
    "hs_blur_down": (_i, [_vp, _i, _i, _i, _vp, _i, _vp]),
    "hs_blur_down_adjoint": (_i, [_vp, _i, _i, _i, _i, _vp, _vp]),
    "hs_upsample2": (_i, [_vp, _i, _vp, _i, _i, _i, _f, _vp]),
    "hs_upsample2_adjoint": (_i, [_vp, _i, _i, _i, _vp, _i, _f, _vp]),
    "hs_warp": (_i, [_vp, _vp, _vp, _i, _i, _i, _vp, _vp]),
    "hs_warp_adjoint_workspace_bytes": (_sz, [_i, _i, _i]),
    "hs_warp_adjoint": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _vp, _sz, _vp]),
    "hs_backward": (_i, [_vp, _i, _i, _i, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz,
                         _cfgp, _vp]),
}

HS_NOALLOC_SCRATCH_BYTES = 48 << 20


def lib():
    """Load libhsflow.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m hindemith_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def status_string(status: int) -> str:
    return lib().hs_status_string(int(status)).decode()


def check(status: int, func: str) -> None:
    if status != HS_OK:
        raise HSError(status, func, lib().hs_last_error().decode())


def make_config(sweeps_per_pass=0, rows_per_segment=0, fast_math=False, avg_edge=0.0,
                avg_corner=0.0, layout=0) -> hs_config:
    c = hs_config()
    c.layout = int(layout)
    c.sweeps_per_pass = int(sweeps_per_pass)
    c.rows_per_segment = int(rows_per_segment)
    c.fast_math = 1 if fast_math else 0
    c.avg_edge = float(avg_edge)
    c.avg_corner = float(avg_corner)
    return c
