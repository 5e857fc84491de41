"""The ``@hm`` decorator -- the reference's user entry point (hindemith.py:14-30).

    from hindemith_b200 import hm, Stencil, defines

    @hm
    def flow(I0, I1, Dx, Dy, Dt, A, alpha2, u, v):
        ...
    u, v = flow(I0=..., I1=..., ...)      # keyword arguments only

On the first call with a given signature the function's source is parsed into a
statement list (``frontend.parse``); later calls with the same signature reuse it.
The signature is the function, every keyword's name, kind, dtype and shape, and the
tuning ``defines`` -- the reference keys on kwarg class names and shapes only
(PyAST.py:155-170).  Results are fresh arrays (the reference hands back views of its
own buffers, which the next call overwrites; backend.cpp:210-243).
"""
from __future__ import annotations

from typing import Any, Dict

import numpy as np

from .frontend import Executor, HMCompileError, function_source, parse, symbol_kind

# Module-global tuning constants, as in the reference (hindemith.py:15).  Keys read here:
#   hs_sweeps_per_pass  -- temporal-blocking depth T of the fused sweep (0 or absent:
#                          autotuned per shape and form, see hs_autotune)
#   hs_rows_per_segment -- rows per warp work item (0 = the tuned or default value)
#   hs_fast_math        -- True: FMA form (within 1e-4); False: bit-identical order
#   hs_autotune         -- False: without hs_sweeps_per_pass, take the library's default
#                          configuration instead of timing candidates on the first call
# The reference's OpenCL launch-geometry keys (nd20, nt20, ne20, ...) are accepted and
# ignored: launch geometry here is chosen per device.
defines: Dict[str, Any] = {}
state: Dict[str, Any] = {}


def _signature(kwargs) -> tuple:
    import torch

    sig = []
    for k in sorted(kwargs):
        v = kwargs[k]
        kind = symbol_kind(v)
        if isinstance(v, np.ndarray):
            sig.append((k, kind, str(v.dtype), v.shape))
        elif isinstance(v, torch.Tensor):
            sig.append((k, kind, str(v.dtype), tuple(v.shape)))
        else:
            sig.append((k, kind, type(v).__name__))
    return tuple(sig)


class hm_fn:
    def __init__(self, fn):
        self.fn = fn
        self.source = function_source(fn)
        self._cache: Dict[tuple, Executor] = {}
        self.__name__ = getattr(fn, "__name__", "hm_fn")
        self.__doc__ = getattr(fn, "__doc__", None)

    def compile(self, **kwargs) -> Executor:
        key = (_signature(kwargs), tuple(sorted((k, repr(v)) for k, v in defines.items())))
        ex = self._cache.get(key)
        if ex is None:
            params = {k: symbol_kind(v) for k, v in kwargs.items()}
            prog = parse(self.source, params)
            ex = Executor(prog, defines)
            self._cache[key] = ex
        return ex

    def __call__(self, *args, **kwargs):
        if args:
            raise HMCompileError("@hm functions take keyword arguments only")
        ex = self.compile(**kwargs)
        before = dict(ex.stats)
        out = ex.run(kwargs)
        # counts of this call alone
        state["last_stats"] = {k: v - before.get(k, 0) for k, v in ex.stats.items()}
        return out


def hm(fn):
    return hm_fn(fn)
