"""Batched Horn-Schunck: many pairs of uneven size in one persistent launch.

    from hindemith_b200.batched import BatchPlan
    plan = BatchPlan([(H, W, alpha, iters), ...], config)   # preallocates everything
    plan.I0[i].copy_(...); plan.I1[i].copy_(...)            # fill the input planes
    plan.capture()                                          # one warm-up run + CUDA graph
    plan.replay()                                           # re-run the whole batch
    u, v = plan.u[i], plan.v[i]

``forward_batched(pairs)`` is the eager one-call form.  Batches larger than the C ABI's
HS_MAX_BATCH (128) are split into consecutive launches with separate workspaces.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib as L
from . import device as D


hs_pair_desc = L.hs_pair_desc
HS_MAX_BATCH = L.HS_MAX_BATCH


def _descs(rows) -> ctypes.Array:
    arr = (hs_pair_desc * len(rows))()
    for d, (I0, I1, u, v, alpha, iters) in zip(arr, rows):
        H, W = I0.shape
        d.I0, d.I1 = I0.data_ptr(), I1.data_ptr()
        d.u, d.v = u.data_ptr(), v.data_ptr()
        d.H, d.W, d.ld = H, W, I0.stride(0)
        d.alpha = float(np.float32(alpha))
        d.iters = int(iters)
        d.reserved = 0
    return arr


def workspace_bytes(specs: Sequence[Tuple[int, int, float, int]], config=None) -> int:
    """Workspace of one launch for (H, W, alpha, iters) specs (host-side, no device)."""
    arr = (hs_pair_desc * len(specs))()
    for d, (H, W, alpha, iters) in zip(arr, specs):
        d.H, d.W, d.ld = H, W, D.padded_ld(W)
        d.alpha, d.iters = float(alpha), int(iters)
    cfg = config if config is not None else L.make_config()
    return int(L.lib().hs_forward_batched_workspace_bytes(arr, len(specs), ctypes.byref(cfg)))


class BatchPlan:
    """Fixed batch: input/output planes, workspace and status preallocated on the device."""

    def __init__(self, specs: Sequence[Tuple[int, int, float, int]], config=None, device=None):
        self.specs = [(int(H), int(W), float(a), int(n)) for H, W, a, n in specs]
        if not self.specs:
            raise ValueError("empty batch")
        self.config = config if config is not None else L.make_config()
        self.device = torch.device(device or "cuda")
        self.I0, self.I1, self.u, self.v = [], [], [], []
        for H, W, _, _ in self.specs:
            planes = D.empty_planes(4, H, W, self.device)
            planes.zero_()
            self.I0.append(planes[0])
            self.I1.append(planes[1])
            self.u.append(planes[2])
            self.v.append(planes[3])
        self.chunks = []
        for c0 in range(0, len(self.specs), HS_MAX_BATCH):
            idx = list(range(c0, min(c0 + HS_MAX_BATCH, len(self.specs))))
            rows = [(self.I0[i], self.I1[i], self.u[i], self.v[i], self.specs[i][2], self.specs[i][3])
                    for i in idx]
            arr = _descs(rows)
            nbytes = L.lib().hs_forward_batched_workspace_bytes(arr, len(idx), ctypes.byref(self.config))
            if nbytes == 0:
                raise L.HSError(L.HS_ERR_INVALID_ARG, "hs_forward_batched_workspace_bytes",
                                "invalid pair description")
            ws = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
            self.chunks.append((arr, len(idx), ws))
        self.status = torch.zeros(len(self.chunks), dtype=torch.int32, device=self.device)
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    @property
    def pixel_iters(self) -> int:
        return sum(H * W * n for H, W, _, n in self.specs)

    def run(self, stream=None) -> None:
        h = D.stream_handle(stream)
        for c, (arr, n, ws) in enumerate(self.chunks):
            st = L.lib().hs_forward_batched(arr, n, D.ptr(ws), ws.numel(), ctypes.byref(self.config),
                                            ctypes.c_void_p(self.status.data_ptr() + 4 * c), h)
            L.check(st, "hs_forward_batched")

    def capture(self) -> torch.cuda.CUDAGraph:
        """Run once (sets kernel attributes), then capture one run into a CUDA graph."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run(s)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.run(s)
        self.graph = g
        return g

    def replay(self) -> None:
        if self.graph is None:
            raise RuntimeError("capture() first")
        self.graph.replay()

    def check(self) -> None:
        """Synchronise and raise if a device-side wait gave up."""
        st = self.status.cpu().tolist()
        for c, code in enumerate(st):
            if code != L.HS_OK:
                raise L.HSError(code, "hs_forward_batched", f"chunk {c}: device status {code}")


def forward_batched(pairs: Sequence[Tuple[torch.Tensor, torch.Tensor, float, int]],
                    config=None, stream=None) -> List[Tuple[torch.Tensor, torch.Tensor]]:
    """Eager batched forward: [(I0, I1, alpha, iters)] -> [(u, v)] planes."""
    specs = [(int(I0.shape[0]), int(I0.shape[1]), a, n) for I0, I1, a, n in pairs]
    with D.stream_scope(stream):  # planes, copies and the launch all on `stream`
        plan = BatchPlan(specs, config, device=pairs[0][0].device if pairs else None)
        for i, (I0, I1, _, _) in enumerate(pairs):
            plan.I0[i].copy_(I0)
            plan.I1[i].copy_(I1)
        plan.run(stream)
    return list(zip(plan.u, plan.v))
