"""Fusion of ``@hm`` statement lists into runtime-compiled CUDA kernels.

The reference's middle end groups statements into fused kernels (fusion.cpp:113-303) by a
dataflow analysis (dataflow.cpp:88-315) and promotes dead intermediates to registers
(lm.cpp:170-276, 467-755).  This pass does the same on the front end's statement list:

* A *group* is a maximal run of consecutive per-pixel statements -- Stencil2DMVM, the
  Array2DOp family, Array2DCopy, sqrt, red/black and sum2d -- with one split rule: a
  stencil may not read an array written earlier in the same group (its neighbours would
  not be materialised yet: the reference splits on the same stencil-read vs
  element-write conflict).  Scalar statements between them are host arithmetic; they
  move to the start of the group unless they read a sum2d of the same group, which ends
  the group.
* Arrays read by the group and defined before it are kernel inputs; arrays written in
  the group are kernel outputs only if something outside the group reads them (or the
  function returns them) -- every other intermediate lives in a register.
* Each group becomes one kernel body (CUDA C) for ``hs_fused_launch``, which compiles
  it with NVRTC for sm_100a and caches it.  Stencil weights and scalar operands are
  kernel parameters, so new values reuse the compiled kernel; tap offsets are part of
  the code.

Semantics are the statement-by-statement FP32 semantics: each operation rounds once
(the kernels compile with -fmad=false unless ``hs_fast_math``), stencils accumulate from
0 in tap order, sum2d accumulates in double and rounds once to float.
"""
from __future__ import annotations

import ctypes
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

from . import _lib as L

FUSABLE = {"Stencil2DMVM", "Array2DOp", "Array2DScalarOp", "ScalarArray2DOp", "Array2DCopy",
           "Array2DSqrt", "RedArray2D", "BlackArray2D", "Array2DSum"}
HOST_SCALAR = {"Const", "ScalarOp", "ScalarNeg", "ScalarCopy", "ScalarSqrt"}
_CSYM = {"Add": "+", "Sub": "-", "Mult": "*", "Div": "/"}


def _reads(s) -> List[str]:
    out = [a for a in s.args if isinstance(a, str)]
    if s.kind == "HSSweeps":
        out += [v for k, v in s.info.items() if k in ("Ix", "Iy", "It", "U", "V", "alpha2", "A")]
    if isinstance(s.ub, str):
        out.append(s.ub)
    return out


def _writes(s) -> List[str]:
    w = [s.dst] if s.dst is not None else []
    w += list(s.info.get("dsts", ()))
    if s.kind == "HSSweeps":
        w += [s.info["U"], s.info["V"]]
    if s.kind in ("SetBroxMatrix", "SetBroxRedblackMatrix"):
        w.append(s.args[0])  # fills the matrix in place
    return w


def _all_reads(stmts, acc: Dict[int, set]) -> set:
    """Names read by every statement, recursively; also records per-statement reads."""
    names = set()
    for s in stmts:
        r = set(_reads(s))
        if s.kind == "Return":
            r |= set(s.args)
        acc[id(s)] = r
        names |= r
        names |= _all_reads(s.body, acc)
    return names


def fuse_program(prog) -> None:
    """Replace runs of fusable statements by "Fused" statements, in every block."""
    per_stmt: Dict[int, set] = {}
    _all_reads(prog.body, per_stmt)
    params = set(prog.params)
    counter = [0]

    def reads_outside(group_ids: set) -> set:
        out = set()
        for sid, r in per_stmt.items():
            if sid not in group_ids:
                out |= r
        return out

    def block(stmts):
        res = []
        i = 0
        while i < len(stmts):
            s = stmts[i]
            if s.body:
                s.body = block(s.body)
            if s.kind not in FUSABLE:
                res.append(s)
                i += 1
                continue
            group, pre, written, sums = [], [], set(), set()  # (position, stmt) lists
            j = i
            while j < len(stmts):
                t = stmts[j]
                if t.kind in HOST_SCALAR:
                    if any(a in sums for a in _reads(t)):
                        break
                    pre.append((j, t))
                    j += 1
                    continue
                if t.kind not in FUSABLE:
                    break
                if t.kind == "Stencil2DMVM" and t.args[1] in written:
                    break
                if any(a in sums for a in _reads(t)):
                    break
                group.append((j, t))
                written.update(_writes(t))
                if t.kind == "Array2DSum":
                    sums.add(t.dst)
                j += 1
            last = group[-1][0]
            hoisted = [t for pos, t in pre if pos < last]
            after = [t for pos, t in pre if pos > last]
            gstmts = [t for _, t in group]
            if len(gstmts) == 1 and gstmts[0].kind == "Array2DCopy":
                res.extend(hoisted + gstmts + after)  # a rebinding needs no kernel
            else:
                live = reads_outside(set(id(t) for t in gstmts)) | params
                res.extend(hoisted)
                res.append(_make_group(gstmts, live, counter))
                res.extend(after)
            i = j
        return res

    prog.body = block(prog.body)


def _make_group(group, live: set, counter):
    from .frontend import Stmt

    counter[0] += 1
    written = []
    for t in group:
        for w in _writes(t):
            if w not in written:
                written.append(w)
    # a name read in the group before the group writes it carries a value across loop
    # iterations: it is an output too
    seen, carried = set(), set()
    for t in group:
        carried |= set(a for a in _reads(t) if a not in seen)
        seen |= set(_writes(t))
    outs = [w for w in written if (w in live or w in carried)
            and not any(t.dst == w and t.kind == "Array2DSum" for t in group)]
    sums = [t.dst for t in group if t.kind == "Array2DSum"]
    return Stmt("Fused", None, (), info={"stmts": group, "outputs": outs, "sums": sums,
                                         "id": counter[0]})


# ------------------------------------------------------------------ code generation

class _Gen:
    def __init__(self, env):
        self.env = env
        self.inputs: List[str] = []     # env names, in input-slot order
        self.scalars: List[float] = []  # parameter values, in slot order
        self.lines: List[str] = []
        self.reg: Dict[str, str] = {}   # array name -> C register holding its pixel value
        self.nreg = 0

    def new_reg(self, expr: str) -> str:
        r = f"r{self.nreg}"
        self.nreg += 1
        self.lines.append(f"const float {r} = {expr};")
        return r

    def input_slot(self, name: str) -> int:
        if name not in self.inputs:
            if len(self.inputs) == L.HS_FUSED_MAX_IN:
                raise _TooBig("inputs")
            self.inputs.append(name)
        return self.inputs.index(name)

    def scalar(self, value) -> str:
        v = np.float32(value)
        for j, w in enumerate(self.scalars):  # equal values share a slot (bitwise)
            if np.float32(w).view(np.uint32) == v.view(np.uint32):
                return f"S({j})"
        if len(self.scalars) == L.HS_FUSED_MAX_SCALARS:
            raise _TooBig("scalars")
        self.scalars.append(float(v))
        return f"S({len(self.scalars) - 1})"

    def value(self, name: str) -> str:
        if name in self.reg:
            return self.reg[name]
        k = self.input_slot(name)
        r = self.new_reg(f"IN({k})")
        self.reg[name] = r
        return r


class _TooBig(Exception):
    pass


def codegen(stmts, outputs, sums, env) -> Tuple[str, "_Gen"]:
    """The kernel body of one group and its argument lists."""
    g = _Gen(env)
    sum_slot = {n: i for i, n in enumerate(sums)}
    for t in stmts:
        k = t.kind
        if k == "Stencil2DMVM":
            st = env[t.args[0]]
            w, ox, oy = st.taps()
            src = g.input_slot(t.args[1])
            acc = f"r{g.nreg}"
            g.nreg += 1
            g.lines.append(f"float {acc} = 0.0f;")
            for wd, dx, dy in zip(w, ox, oy):
                g.lines.append(f"{acc} = {acc} + {g.scalar(wd)} * LD({src}, {int(dx)}, {int(dy)});")
            g.reg[t.dst] = acc
        elif k == "Array2DOp":
            a, b = g.value(t.args[0]), g.value(t.args[1])
            g.reg[t.dst] = g.new_reg(f"{a} {_CSYM[t.op]} {b}")
        elif k == "Array2DScalarOp":
            a = g.value(t.args[0])
            g.reg[t.dst] = g.new_reg(f"{a} {_CSYM[t.op]} {g.scalar(env[t.args[1]])}")
        elif k == "ScalarArray2DOp":
            b = g.value(t.args[1])
            g.reg[t.dst] = g.new_reg(f"{g.scalar(env[t.args[0]])} {_CSYM[t.op]} {b}")
        elif k == "Array2DCopy":
            g.reg[t.dst] = g.value(t.args[0])
        elif k == "Array2DSqrt":
            g.reg[t.dst] = g.new_reg(f"sqrtf({g.value(t.args[0])})")
        elif k == "RedArray2D":  # RedArray2D.cpp:26
            g.reg[t.dst] = g.new_reg(f"((X + Y) & 1) ? 0.0f : {g.value(t.args[0])}")
        elif k == "BlackArray2D":  # BlackArray2D.cpp:26
            g.reg[t.dst] = g.new_reg(f"((X + Y) & 1) ? {g.value(t.args[0])} : 0.0f")
        elif k == "Array2DSum":
            g.lines.append(f"SUM({sum_slot[t.dst]}, {g.value(t.args[0])});")
        else:
            raise AssertionError(f"not fusable: {k}")
    if len(outputs) > L.HS_FUSED_MAX_OUT:
        raise _TooBig("outputs")
    for j, name in enumerate(outputs):
        g.lines.append(f"OUT({j}) = {g.value(name)};")
    return "\n".join(g.lines) + "\n", g


def run_group(stmt, env, fast_math: bool, stats: Dict[str, int]) -> bool:
    """Execute one Fused statement: generate, launch, bind outputs and sums in env.
    False when the group exceeds the kernel's argument limits (the caller then runs its
    statements one operator each)."""
    import torch

    from . import device as D

    info = stmt.info
    # the generated body depends on the stencils' taps and the scalar operands' values only
    # (inputs, outputs and their order are fixed by the statements): cache it per value set
    key = _value_signature(info["stmts"], env)
    cache = info.setdefault("codegen_cache", {})
    hit = cache.get(key)
    if hit is None:
        try:
            body, g = codegen(info["stmts"], info["outputs"], info["sums"], env)
        except _TooBig:
            stats["fused_fallback"] = stats.get("fused_fallback", 0) + 1
            return False
        hit = (body.encode(), list(g.inputs), list(g.scalars))
        if len(cache) < 64:
            cache[key] = hit
    body_b, inputs, scalars = hit
    planes = D._same_layout(*(env[n] for n in inputs)) if inputs else ()
    if planes:
        H, W = planes[0].shape
        ld = planes[0].stride(0)
        dev = planes[0].device
        for p in planes:
            if p.shape != (H, W):
                raise ValueError(f"fused statements mix shapes {tuple(p.shape)} and {(H, W)}")
    else:
        raise ValueError("a fused group needs at least one array input")
    args = L.hs_fused_args()
    for k, p in enumerate(planes):
        args.in_[k] = p.data_ptr()
    outs = torch.empty((max(1, len(info["outputs"])), H, ld), dtype=torch.float32, device=dev)
    for j in range(len(info["outputs"])):
        args.out[j] = outs[j].data_ptr()
    for j, v in enumerate(scalars):
        args.s[j] = v
    args.H, args.W, args.ld = H, W, ld
    nsums = len(info["sums"])
    args.nsums = nsums
    lib = L.lib()
    sums_dev = ws = None
    if nsums:
        sums_dev = torch.empty(nsums, dtype=torch.float64, device=dev)
        args.sums = sums_dev.data_ptr()
        ws = torch.empty(int(lib.hs_fused_workspace_bytes(H, W, nsums)), dtype=torch.uint8, device=dev)
    L.check(lib.hs_fused_launch(body_b, 1 if fast_math else 0, ctypes.byref(args),
                                D.ptr(ws) if ws is not None else None,
                                ws.numel() if ws is not None else 0, D.stream_handle()),
            "hs_fused_launch")
    stats["fused_launches"] = stats.get("fused_launches", 0) + 1
    for j, name in enumerate(info["outputs"]):
        env[name] = outs[j][:, :W]
    if nsums:
        vals = sums_dev.cpu().numpy()
        for j, name in enumerate(info["sums"]):
            env[name] = np.float32(vals[j])
    return True


def _value_signature(stmts, env) -> tuple:
    parts = []
    for t in stmts:
        if t.kind == "Stencil2DMVM":
            w, ox, oy = env[t.args[0]].taps()
            parts.append((w.tobytes(), ox.tobytes(), oy.tobytes()))
        elif t.kind == "Array2DScalarOp":
            parts.append(np.float32(env[t.args[1]]).tobytes())
        elif t.kind == "ScalarArray2DOp":
            parts.append(np.float32(env[t.args[0]]).tobytes())
    return tuple(parts)


def split_group(stmt):
    """One Fused statement per member statement (for a group over the argument limits):
    every array it writes is an output."""
    from .frontend import Stmt

    out = []
    for t in stmt.info["stmts"]:
        outs = [w for w in _writes(t) if t.kind != "Array2DSum"]
        sums = [t.dst] if t.kind == "Array2DSum" else []
        out.append(Stmt("Fused", None, (), info={"stmts": [t], "outputs": outs, "sums": sums,
                                                 "id": stmt.info["id"]}))
    return out
