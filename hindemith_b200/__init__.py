"""hindemith_b200 -- a B200 (sm_100a) implementation of Hindemith's structured-grid
stencil and Horn-Schunck optical-flow path.

User surface (the reference's): ``hm``, ``defines``, ``Stencil``.
Device API (torch CUDA tensors): ``hs_forward``, ``hs_sweeps``, ``hs_derivs``,
``stencil2d`` and the pointwise Array2D operators in ``hindemith_b200.device``.
The compute is libhsflow.so (hindemith_b200/_lib), a C-ABI CUDA library.
"""
from .hindemith import defines, hm, hm_fn, state  # noqa: F401
from .hlib import SpMat2D, Stencil, brox_offsets, hs_average_stencil, hs_derivative_stencils  # noqa: F401
from ._lib import HSError, hs_config, make_config  # noqa: F401


def __getattr__(name):
    # device-level entry points load torch lazily
    if name in ("hs_forward", "hs_sweeps", "hs_derivs", "stencil2d"):
        from . import device
        return getattr(device, name)
    raise AttributeError(name)
