"""Python-side types of the Hindemith surface: ``Stencil`` and the canonical HS stencils.

``Stencil(data, offx, offy)`` keeps the reference's constructor and attributes
(hlib.py:166-171): ``data`` holds the tap weights, ``offx`` / ``offy`` the integer
x (width) and y (height) offsets, one entry per tap, and ``dtype`` is ``data.dtype``.
Its product with a 2-D array is the clamp-to-edge stencil of
Operations/StructuredGrid/Stencil2DMVM.cpp:34-59, computed by libhsflow on the GPU:
the reference's NumPy ``Stencil.__mul__`` (hlib.py:173-191, edge padding) gives the
same values for symmetric stencils and raises for asymmetric ones; this version
accepts any tap set.
"""
from __future__ import annotations

import numpy as np


class Stencil:
    def __init__(self, data, offx, offy):
        self.data = np.asarray(data)
        self.offx = np.asarray(offx)
        self.offy = np.asarray(offy)
        self.dtype = self.data.dtype
        if not (len(self.data) == len(self.offx) == len(self.offy)):
            raise ValueError("Stencil data, offx and offy must have one entry per tap")

    @property
    def ndiags(self) -> int:
        return len(self.data)

    def taps(self):
        """(weights float32, offx int32, offy int32) as the C ABI takes them."""
        return (np.ascontiguousarray(self.data, dtype=np.float32),
                np.ascontiguousarray(self.offx, dtype=np.int32),
                np.ascontiguousarray(self.offy, dtype=np.int32))

    def __mul__(self, b):
        from . import device
        import torch

        w, ox, oy = self.taps()
        if isinstance(b, np.ndarray):
            out = device.stencil2d(w, ox, oy, device.as_plane(b))
            return out.cpu().numpy().astype(b.dtype, copy=False)
        if isinstance(b, torch.Tensor):
            return device.stencil2d(w, ox, oy, device.as_plane(b))
        return NotImplemented

    def __repr__(self):
        return f"Stencil(ndiags={self.ndiags}, dtype={self.dtype})"


class SpMat2D:
    """A sparse 2-D grid operator in diagonal form, the reference's SpMat2D
    (hlib.py:140-146): `data` (ndiags, H, W), one plane per diagonal, and the diagonal
    offsets `offx`, `offy`.  On the device each diagonal is indexed by the column of its
    entry (SpmvDIA2D.cpp:36-45, SetBroxMatrix.cpp:38-80)."""

    def __init__(self, data, offx, offy):
        self.data = data
        self.offx = np.asarray(offx)
        self.offy = np.asarray(offy)
        self.ndiags, self.dim0, self.dim1 = tuple(data.shape)
        self.dtype = data.dtype
        if not (self.ndiags == len(self.offx) == len(self.offy)):
            raise ValueError("SpMat2D data, offx and offy must have one entry per diagonal")

    def __repr__(self):
        return f"SpMat2D(ndiags={self.ndiags}, {self.dim0}x{self.dim1})"


def brox_offsets():
    """Diagonal offsets of the Brox smoothness matrix: top, left, mid, right, bottom."""
    return (np.array([0, -1, 0, 1, 0], dtype=np.int32), np.array([-1, 0, 0, 0, 1], dtype=np.int32))


def hs_average_stencil() -> Stencil:
    """The Horn-Schunck 3x3 average: 1/12 at the corners, 1/6 at the edges, no centre;
    taps in row-major order."""
    offx = np.array([-1, 0, 1, -1, 1, -1, 0, 1], dtype=np.int32)
    offy = np.array([-1, -1, -1, 0, 0, 1, 1, 1], dtype=np.int32)
    w = np.where((offx != 0) & (offy != 0), np.float32(1 / 12), np.float32(1 / 6)).astype(np.float32)
    return Stencil(w, offx, offy)


def hs_derivative_stencils():
    """(Dx, Dy, Dt): the 2x2x2 first-difference stencils over the {0,1}^2 block."""
    offx = np.array([0, 1, 0, 1], dtype=np.int32)
    offy = np.array([0, 0, 1, 1], dtype=np.int32)
    dx = Stencil(np.array([-0.25, 0.25, -0.25, 0.25], dtype=np.float32), offx, offy)
    dy = Stencil(np.array([-0.25, -0.25, 0.25, 0.25], dtype=np.float32), offx, offy)
    dt = Stencil(np.array([0.25, 0.25, 0.25, 0.25], dtype=np.float32), offx, offy)
    return dx, dy, dt


def hs_average_weights(st: Stencil):
    """(edge, corner) weights if `st` is a symmetric 3x3 average whose taps run in
    row-major order (an optional centre tap must weigh 0); else None."""
    w, ox, oy = st.taps()
    taps = list(zip(ox.tolist(), oy.tolist(), w.tolist()))
    order = [(dx, dy) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    with_centre = [(dx, dy) for (dx, dy) in order]
    without = [(dx, dy) for (dx, dy) in order if (dx, dy) != (0, 0)]
    pos = [(a, b) for a, b, _ in taps]
    if pos == without:
        pass
    elif pos == with_centre:
        if taps[4][2] != 0.0:
            return None
    else:
        return None
    edge = [c for a, b, c in taps if (a == 0) != (b == 0)]
    corner = [c for a, b, c in taps if a != 0 and b != 0]
    if len(set(edge)) != 1 or len(set(corner)) != 1:
        return None
    return np.float32(edge[0]), np.float32(corner[0])
