"""Front-end compiler of the ``@hm`` surface: Python AST -> statement list -> CUDA calls.

It accepts the operation set the reference's templates accept on this path
(Templates.py): ``Stencil * Array2D`` (Stencil2DMVM, :601-617), ``Array2D op Array2D``
(Array2DOp, :103-120), ``Array2D op Scalar`` (Array2DScalarOp, :141-158), ``Scalar op
Array2D`` (ScalarArray2DOp, :179-196), ``Scalar op Scalar`` (ScalarOp, :238-255),
assignment and tuple assignment (Array2DCopy, :668-696), ``for _ in range(N)``
(Iterator, :57-71) and ``return a`` / ``return a, b`` (Return, :760-780; Tuple,
:891-902).  The symbol table is built from the call's keyword arguments the way
``PrototypeVisitor`` does (PyAST.py:16-41): 2-D arrays become Array2D, ``Stencil``
objects Stencil, NumPy float32/float64/int64 scalars Scalar.

Lowering.  Every statement has a direct CUDA operator in libhsflow, so any accepted
program runs on the device one operator per statement (the reference's unfused
semantics).  On top of that the compiler recognises the Horn-Schunck Jacobi loop --
the composition fusion.cpp/dataflow.cpp turn into two fused kernels per sweep -- and
replaces the whole loop by one ``hs_sweeps`` call: T sweeps per HBM pass in one
kernel, bit-identical to the statement-by-statement result.  Recognition is
structural (operands may commute, sums may not re-associate) and is re-checked
against the stencil's values at run time; a loop that does not match runs unfused.

Scalar-by-scalar statements fold on the host in IEEE FP32 (NumPy float32), which is
what the reference's one-thread ScalarOp kernel computes.
"""
from __future__ import annotations

import ast
import inspect
import itertools
import textwrap
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

from . import _lib as L
from .hlib import Stencil, hs_average_weights

ARRAY2D, STENCIL, SCALAR, ARRAY3D, SPMAT2D = "Array2D", "Stencil", "Scalar", "Array3D", "SpMat2D"
_OPS = {ast.Add: "Add", ast.Sub: "Sub", ast.Mult: "Mult", ast.Div: "Div"}


class HMCompileError(TypeError):
    """The function uses a construct the Hindemith surface does not support."""


def _call_name(node) -> str:
    if not isinstance(node.func, ast.Name):
        raise HMCompileError("only calls of plain function names are supported")
    return node.func.id


# ------------------------------------------------------------------ IR

@dataclass
class Stmt:
    kind: str                 # Stencil2DMVM, Array2DOp, Array2DScalarOp, ScalarArray2DOp,
                              # ScalarOp, Array2DCopy, ScalarCopy, Iterator, Return, HSSweeps
    dst: Optional[str] = None
    args: Tuple = ()
    op: Optional[str] = None
    body: List["Stmt"] = field(default_factory=list)
    ub: Any = None            # Iterator bound: int or kwarg name
    info: Dict[str, Any] = field(default_factory=dict)


@dataclass
class Program:
    name: str
    params: Dict[str, str]    # kwarg name -> kind
    body: List[Stmt]


def symbol_kind(obj) -> str:
    """Kind of a keyword argument, as PrototypeVisitor.visit_FunctionDef assigns it."""
    import torch

    if isinstance(obj, Stencil) or type(obj).__name__ == "Stencil":
        return STENCIL
    if type(obj).__name__ in ("SpMat2D", "DeviceSpMat2D"):
        return SPMAT2D
    if isinstance(obj, np.ndarray):
        if obj.ndim == 2:
            return ARRAY2D
        raise HMCompileError(f"only 2-D arrays are supported on this path, got {obj.ndim}-D")
    if isinstance(obj, torch.Tensor):
        if obj.dim() == 2:
            return ARRAY2D
        raise HMCompileError(f"only 2-D tensors are supported on this path, got {obj.dim()}-D")
    if isinstance(obj, (np.float32, np.float64, np.int64, float, int)):
        return SCALAR
    raise HMCompileError(f"unsupported argument type {type(obj).__name__}")


class _Compiler:
    def __init__(self, params: Dict[str, str]):
        self.kinds: Dict[str, str] = dict(params)
        self.tmp = itertools.count()

    def fresh(self) -> str:
        return f"_f{next(self.tmp)}"

    def expr(self, node, out: List[Stmt]) -> Tuple[str, str]:
        """Compile an expression; returns (name, kind).  Sub-expressions are emitted
        post-order into `out`, as EmitVisitor does (PyAST.py:52-58)."""
        if isinstance(node, ast.Name):
            if node.id not in self.kinds:
                raise HMCompileError(f"name '{node.id}' is not an argument or assigned before use")
            return node.id, self.kinds[node.id]
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)) \
                and not isinstance(node.value, bool):
            name = self.fresh()
            out.append(Stmt("Const", name, (np.float32(node.value),)))
            self.kinds[name] = SCALAR
            return name, SCALAR
        if isinstance(node, ast.UnaryOp) and isinstance(node.op, ast.USub):
            a, ka = self.expr(node.operand, out)
            name = self.fresh()
            if ka == ARRAY2D:
                zero = self.fresh()
                out.append(Stmt("Const", zero, (np.float32(0.0),)))
                self.kinds[zero] = SCALAR
                out.append(Stmt("ScalarArray2DOp", name, (zero, a), op="Sub"))
                self.kinds[name] = ARRAY2D
            elif ka == SCALAR:
                out.append(Stmt("ScalarNeg", name, (a,)))
                self.kinds[name] = SCALAR
            else:
                raise HMCompileError("unary minus of a Stencil is not supported")
            return name, self.kinds[name]
        if isinstance(node, ast.BinOp):
            op = _OPS.get(type(node.op))
            if op is None:
                raise HMCompileError(f"operator {type(node.op).__name__} is not supported")
            a, ka = self.expr(node.left, out)
            b, kb = self.expr(node.right, out)
            name = self.fresh()
            if ka == STENCIL and kb == ARRAY2D and op == "Mult":
                out.append(Stmt("Stencil2DMVM", name, (a, b)))
                kind = ARRAY2D
            elif ka == SPMAT2D and kb == ARRAY2D and op == "Mult":  # Templates.py:583-599
                out.append(Stmt("SpmvDIA2D", name, (a, b)))
                kind = ARRAY2D
            elif ka == ARRAY2D and kb == ARRAY2D:
                out.append(Stmt("Array2DOp", name, (a, b), op=op))
                kind = ARRAY2D
            elif ka == ARRAY2D and kb == SCALAR:
                out.append(Stmt("Array2DScalarOp", name, (a, b), op=op))
                kind = ARRAY2D
            elif ka == SCALAR and kb == ARRAY2D:
                out.append(Stmt("ScalarArray2DOp", name, (a, b), op=op))
                kind = ARRAY2D
            elif ka == SCALAR and kb == SCALAR:
                out.append(Stmt("ScalarOp", name, (a, b), op=op))
                kind = SCALAR
            else:
                raise HMCompileError(f"no operation matches {ka} {op} {kb}")
            self.kinds[name] = kind
            return name, kind
        if isinstance(node, ast.Call):
            names, kinds = self.call(node, out)
            if len(names) != 1:
                raise HMCompileError(f"{_call_name(node)}() returns {len(names)} values: assign them "
                                     "to a tuple")
            return names[0], kinds[0]
        if isinstance(node, ast.Tuple):
            raise HMCompileError("tuples are only supported in assignments and returns")
        raise HMCompileError(f"unsupported expression {type(node).__name__}")

    def call(self, node, out: List[Stmt]) -> Tuple[List[str], List[str]]:
        """The reference's call templates (Templates.py): sqrt (:485-534), sum2d (:468-483),
        red / black (:536-568), warp_img2d (:258-275), applyHSPreconditioner (:412-443) and
        hs_matrix_powers (:277-300).  Returns the result names and kinds."""
        fname = _call_name(node)
        if node.keywords:
            raise HMCompileError(f"{fname}() takes positional arguments only")
        args = [self.expr(a, out) for a in node.args]
        kinds = [k for _, k in args]
        names = [n for n, _ in args]

        def want(sig):
            if kinds != list(sig):
                raise HMCompileError(f"{fname}({', '.join(kinds)}): expected ({', '.join(sig)})")

        def one(kind, stmt_kind, **kw):
            name = self.fresh()
            out.append(Stmt(stmt_kind, name, tuple(names), **kw))
            self.kinds[name] = kind
            return [name], [kind]

        if fname == "sqrt":
            if kinds == [ARRAY2D]:
                return one(ARRAY2D, "Array2DSqrt")
            if kinds == [SCALAR]:
                return one(SCALAR, "ScalarSqrt")
            want([ARRAY2D])
        if fname in ("sum2d", "sum"):
            want([ARRAY2D])
            return one(SCALAR, "Array2DSum")
        if fname in ("red", "black"):
            want([ARRAY2D])
            return one(ARRAY2D, "RedArray2D" if fname == "red" else "BlackArray2D")
        if fname == "warp_img2d":
            want([ARRAY2D] * 3)
            return one(ARRAY2D, "WarpImg2D")
        if fname == "set_brox_redblack_matrix":  # Templates.py:332-350
            want([SPMAT2D, ARRAY2D, SCALAR])
            return one(ARRAY2D, "SetBroxRedblackMatrix")
        if fname in ("applyHSPreconditioner", "hs_matrix_powers", "applyBroxPreconditioner",
                     "lk_least_squares"):
            if fname == "applyHSPreconditioner":
                want([STENCIL] + [ARRAY2D] * 5)
                kind, res = "ApplyHSPreconditioner", ARRAY2D
            elif fname == "applyBroxPreconditioner":  # Templates.py:377-410
                want([SPMAT2D] + [ARRAY2D] * 5)
                kind, res = "ApplyBroxPreconditioner", ARRAY2D
            elif fname == "lk_least_squares":  # Templates.py:352-375
                want([ARRAY2D] * 3)
                kind, res = "LKLeastSquares", ARRAY2D
            else:
                want([SCALAR, ARRAY2D, ARRAY2D, ARRAY2D, ARRAY2D])
                kind, res = "HSMatrixPowers", ARRAY3D
            dsts = (self.fresh(), self.fresh())
            out.append(Stmt(kind, None, tuple(names), info={"dsts": dsts}))
            for d in dsts:
                self.kinds[d] = res
            return list(dsts), [res, res]
        raise HMCompileError(f"unsupported call {fname}()")

    def assign(self, targets, value, out: List[Stmt]) -> None:
        if len(targets) != 1:
            raise HMCompileError("chained assignment is not supported")
        tgt = targets[0]
        if isinstance(tgt, ast.Tuple) and isinstance(value, ast.Call):
            names, kinds = self.call(value, out)
            if len(names) != len(tgt.elts):
                raise HMCompileError(f"{_call_name(value)}() returns {len(names)} values, "
                                     f"{len(tgt.elts)} targets given")
            for t, name, kind in zip(tgt.elts, names, kinds):
                self._bind(t, name, kind, out)
            return
        if isinstance(tgt, ast.Tuple):
            if not isinstance(value, ast.Tuple) or len(value.elts) != len(tgt.elts):
                raise HMCompileError("tuple assignment needs a tuple of the same length")
            vals = []
            for v in value.elts:  # every right-hand side is read before any target is bound
                name, kind = self.expr(v, out)
                if isinstance(v, ast.Name) and kind != STENCIL:
                    snap = self.fresh()
                    out.append(Stmt("Array2DCopy" if kind == ARRAY2D else "ScalarCopy", snap, (name,)))
                    self.kinds[snap] = kind
                    name = snap
                vals.append((name, kind))
            for t, (name, kind) in zip(tgt.elts, vals):
                self._bind(t, name, kind, out)
        else:
            name, kind = self.expr(value, out)
            self._bind(tgt, name, kind, out)

    def _bind(self, tgt, name, kind, out):
        if not isinstance(tgt, ast.Name):
            raise HMCompileError("assignment targets must be plain names")
        if kind == STENCIL:
            raise HMCompileError("Stencils cannot be assigned")
        prev = self.kinds.get(tgt.id)
        if prev is not None and prev != kind:
            raise HMCompileError(f"'{tgt.id}' changes kind from {prev} to {kind}")
        copy = {ARRAY2D: "Array2DCopy", SCALAR: "ScalarCopy", ARRAY3D: "Array3DCopy"}[kind]
        out.append(Stmt(copy, tgt.id, (name,)))
        self.kinds[tgt.id] = kind

    def block(self, stmts, out: List[Stmt]) -> None:
        for s in stmts:
            if isinstance(s, ast.Assign):
                self.assign(s.targets, s.value, out)
            elif isinstance(s, ast.For):
                it = s.iter
                if not (isinstance(it, ast.Call) and isinstance(it.func, ast.Name)
                        and it.func.id in ("range", "xrange") and len(it.args) == 1):
                    raise HMCompileError("only `for _ in range(N)` loops are supported")
                arg = it.args[0]
                if isinstance(arg, ast.Constant) and isinstance(arg.value, int):
                    ub = int(arg.value)
                elif isinstance(arg, ast.Name) and self.kinds.get(arg.id) == SCALAR:
                    ub = arg.id
                else:
                    raise HMCompileError("the loop bound must be an integer literal or argument")
                if s.orelse:
                    raise HMCompileError("for/else is not supported")
                body: List[Stmt] = []
                self.block(s.body, body)
                out.append(Stmt("Iterator", body=body, ub=ub))
            elif isinstance(s, ast.Return):
                if s.value is None:
                    out.append(Stmt("Return", args=()))
                    continue
                vals = s.value.elts if isinstance(s.value, ast.Tuple) else [s.value]
                names = tuple(self.expr(v, out)[0] for v in vals)
                out.append(Stmt("Return", args=names, info={"tuple": isinstance(s.value, ast.Tuple)}))
            elif isinstance(s, ast.Expr) and isinstance(s.value, ast.Constant):
                continue  # docstring
            elif (isinstance(s, ast.Expr) and isinstance(s.value, ast.Call)
                  and isinstance(s.value.func, ast.Name) and s.value.func.id == "set_brox_matrix"):
                # Templates.py:311-330: a statement that fills the matrix in place
                args = [self.expr(a, out) for a in s.value.args]
                if [k for _, k in args] != [SPMAT2D, ARRAY2D, SCALAR]:
                    raise HMCompileError("set_brox_matrix(SpMat2D, Array2D, Scalar) expected")
                out.append(Stmt("SetBroxMatrix", None, tuple(n for n, _ in args)))
            elif isinstance(s, ast.Pass):
                continue
            else:
                raise HMCompileError(f"unsupported statement {type(s).__name__}")


def parse(source: str, params: Dict[str, str]) -> Program:
    tree = ast.parse(textwrap.dedent(source))
    fdefs = [n for n in tree.body if isinstance(n, ast.FunctionDef)]
    if len(fdefs) != 1:
        raise HMCompileError("expected exactly one function definition")
    fd = fdefs[0]
    c = _Compiler(params)
    body: List[Stmt] = []
    c.block(fd.body, body)
    prog = Program(fd.name, dict(params), body)
    lower_hs_loops(prog)
    return prog


# ------------------------------------------------------------------ HS loop recognition

def _leaf(name):
    return ("leaf", name)


def _symbolic(body: List[Stmt], env: Dict[str, Any]) -> Optional[Dict[str, Any]]:
    """Expression trees of every name assigned in `body`, over the loop-entry values."""
    env = dict(env)
    for s in body:
        k = s.kind
        get = lambda n: env.get(n, _leaf(n))  # noqa: E731
        if k == "Stencil2DMVM":
            env[s.dst] = ("stencil", s.args[0], get(s.args[1]))
        elif k in ("Array2DOp", "Array2DScalarOp", "ScalarArray2DOp", "ScalarOp"):
            env[s.dst] = ("op", s.op, get(s.args[0]), get(s.args[1]))
        elif k in ("Array2DCopy", "ScalarCopy"):
            env[s.dst] = get(s.args[0])
        elif k == "Const":
            env[s.dst] = ("const", float(s.args[0]))
        else:
            return None  # nested loops, returns: not a plain sweep body
    return env


def _is_op(e, op):
    return isinstance(e, tuple) and e[0] == "op" and e[1] == op


def _comm(e, op):
    """Both operand orders of a commutative node, or [] if `e` is not that op."""
    if not _is_op(e, op):
        return []
    return [(e[2], e[3]), (e[3], e[2])]


def _canon(e):
    """Canonical form: operands of + and * sorted (IEEE + and * commute exactly;
    association is kept, so canonical equality implies bit-identical results)."""
    if isinstance(e, tuple) and e[0] == "op":
        a, b = _canon(e[2]), _canon(e[3])
        if e[1] in ("Add", "Mult") and repr(b) < repr(a):
            a, b = b, a
        return ("op", e[1], a, b)
    if isinstance(e, tuple) and e[0] == "stencil":
        return ("stencil", e[1], _canon(e[2]))
    return e


def _split_mult(e):
    """Mult(x, t) with t a Div node -> (x, t)."""
    if not _is_op(e, "Mult"):
        return None
    if _is_op(e[3], "Div"):
        return e[2], e[3]
    if _is_op(e[2], "Div"):
        return e[3], e[2]
    return None


def _match_hs_body(final: Dict[str, Any], assigned, invariant):
    """Yield every (U, V) with U' = A*U - Ix*t, V' = A*V - Iy*t,
    t = ((Ix*(A*U) + Iy*(A*V)) + It) / den, all of Ix, Iy, It, den loop-invariant.
    The update is symmetric in (U, Ix) <-> (V, Iy); the caller picks the orientation
    whose denominator association matches the kernel's."""
    arrays = sorted(n for n in assigned if isinstance(final.get(n), tuple))
    for U, V in itertools.permutations(arrays, 2):
        eu, ev = final[U], final[V]
        if not (_is_op(eu, "Sub") and _is_op(ev, "Sub")):
            continue
        su, sv = eu[2], ev[2]
        if not (su[0] == "stencil" and su[2] == _leaf(U) and sv[0] == "stencil"
                and sv[2] == _leaf(V) and su[1] == sv[1]):
            continue
        pu, pv = _split_mult(eu[3]), _split_mult(ev[3])
        if pu is None or pv is None:
            continue
        (ix, tu), (iy, tv) = pu, pv
        if _canon(tu) != _canon(tv):
            continue
        num, den = tu[2], tu[3]
        leaves = (ix, iy, den)
        if not all(x[0] == "leaf" and x[1] in invariant for x in leaves):
            continue
        if not (_is_op(num, "Add")):
            continue
        it = num[3] if num[3][0] == "leaf" else num[2]
        if not (it[0] == "leaf" and it[1] in invariant):
            continue
        want = ("op", "Add", ("op", "Add", ("op", "Mult", ix, su), ("op", "Mult", iy, sv)), it)
        if _canon(num) != _canon(want):
            continue
        yield {"U": U, "V": V, "A": su[1], "Ix": ix[1], "Iy": iy[1], "It": it[1],
               "den": den[1]}


def _match_den(expr, ix, iy) -> Optional[str]:
    """den = (alpha2 + Ix*Ix) + Iy*Iy with alpha2 a scalar leaf; returns its name."""
    sq = lambda e, n: _is_op(e, "Mult") and e[2] == _leaf(n) and e[3] == _leaf(n)  # noqa: E731
    for inner, last in _comm(expr, "Add"):
        if not sq(last, iy):
            continue
        for a2, first in _comm(inner, "Add"):
            if sq(first, ix) and a2[0] == "leaf":
                return a2[1]
    return None


def _names_read_after(stmts: List[Stmt]) -> set:
    used = set()
    for s in stmts:
        used.update(a for a in s.args if isinstance(a, str))
        if isinstance(s.ub, str):
            used.add(s.ub)
        used |= _names_read_after(s.body)
    return used


def _assigned(stmts: List[Stmt]) -> List[str]:
    out = []
    for s in stmts:
        if s.dst is not None:
            out.append(s.dst)
        out.extend(_assigned(s.body))
    return out


def lower_hs_loops(prog: Program) -> None:
    """Replace each Horn-Schunck Jacobi Iterator of the top-level block by HSSweeps."""
    body = prog.body
    for i, s in enumerate(body):
        if s.kind != "Iterator":
            continue
        loop_assigned = set(_assigned(s.body))
        final = _symbolic(s.body, {})
        if final is None:
            continue
        before = body[:i]
        top_assigned = _assigned(before)
        counts = {n: top_assigned.count(n) for n in set(top_assigned)}
        invariant = {n for n in (set(prog.params) | set(top_assigned)) if n not in loop_assigned}
        live_after = _names_read_after(body[i + 1:])
        pre = _symbolic(before, {})
        chosen = None
        for m in _match_hs_body(final, loop_assigned, invariant):
            # den must be defined once before the loop as (alpha2 + Ix*Ix) + Iy*Iy
            if counts.get(m["den"], 0) != 1 or any(counts.get(m[k], 0) > 1 for k in ("Ix", "Iy", "It")):
                continue
            if pre is None or m["den"] not in pre:
                continue
            # the den expression refers to Ix, Iy by their own names
            den_expr = _resolve_names(before, m["den"], {m["Ix"], m["Iy"]})
            alpha2 = _match_den(den_expr, m["Ix"], m["Iy"])
            if alpha2 is None:
                continue
            # every other name the loop assigns must be dead after it
            if any(n in live_after for n in loop_assigned if n not in (m["U"], m["V"])):
                continue
            m["alpha2"] = alpha2
            chosen = m
            break
        if chosen is None:
            continue
        m = chosen
        body[i] = Stmt("HSSweeps", info=m, ub=s.ub, body=s.body)


def _resolve_names(stmts: List[Stmt], name: str, stop: set):
    """Expression of `name` after `stmts`, expanding temporaries but keeping the names
    in `stop` (and arguments / scalars) as leaves."""
    defs = {}
    for s in stmts:
        if s.dst is not None:
            defs[s.dst] = s

    def ex(n, depth=0):
        if depth > 64 or n in stop or n not in defs:
            return _leaf(n)
        s = defs[n]
        if s.kind in ("Array2DCopy", "ScalarCopy"):
            return ex(s.args[0], depth + 1)
        if s.kind in ("Array2DOp", "ScalarArray2DOp", "Array2DScalarOp"):
            return ("op", s.op, ex(s.args[0], depth + 1), ex(s.args[1], depth + 1))
        return _leaf(n)

    return ex(name)


# ------------------------------------------------------------------ execution

class Executor:
    """Runs a Program on the current CUDA device (execute.cpp's role)."""

    def __init__(self, prog: Program, defines: Dict[str, Any]):
        from .fusion import fuse_program

        self.prog = prog
        self.defines = dict(defines)
        self.stats = {"hs_sweeps_calls": 0, "unfused_loops": 0, "fused_launches": 0}
        self.last_sweep_config = None  # (depth, rows per segment, layout, fast) of the last HS loop
        if self.defines.get("hs_fuse", True):
            fuse_program(self.prog)

    def config(self) -> L.hs_config:
        d = self.defines
        return L.make_config(sweeps_per_pass=int(d.get("hs_sweeps_per_pass", 0)),
                             rows_per_segment=int(d.get("hs_rows_per_segment", 0)),
                             fast_math=bool(d.get("hs_fast_math", False)))

    def run(self, kwargs: Dict[str, Any]):
        from . import device
        import torch

        env: Dict[str, Any] = {}
        for name, kind in self.prog.params.items():
            val = kwargs[name]
            if kind == ARRAY2D:
                env[name] = device.as_plane(val)
            elif kind == SCALAR:
                env[name] = val if isinstance(val, (np.integer, int)) else np.float32(val)
            elif kind == SPMAT2D:
                from .flow import DeviceSpMat2D

                env[name] = val if isinstance(val, DeviceSpMat2D) else DeviceSpMat2D.from_host(val)
            else:
                env[name] = val
        args = [v for v in kwargs.values() if isinstance(v, torch.Tensor)]
        args += [env[n] for n, k in self.prog.params.items() if k == ARRAY2D]
        handed = {_span(t) for t in args}  # memory the caller holds
        ret = self._block(self.prog.body, env)
        if ret is None:
            return None
        names, is_tuple = ret
        want_numpy = any(isinstance(kwargs[n], np.ndarray) for n, k in self.prog.params.items()
                         if k == ARRAY2D)
        outs = []
        for n in names:
            v = env[n]
            if isinstance(v, torch.Tensor):
                if want_numpy:
                    v = v.cpu().numpy()  # a new host array
                else:
                    # values computed by this call are new tensors and are handed out as they
                    # are; an argument, or a value already handed out, is copied
                    sp = _span(v)
                    if any(_overlap(sp, h) for h in handed):
                        v = v.clone()
                        sp = _span(v)
                    handed.add(sp)
            outs.append(v)
        return tuple(outs) if is_tuple else outs[0]

    def _block(self, stmts: List[Stmt], env):
        for s in stmts:
            r = self._stmt(s, env)
            if r is not None:
                return r
        return None

    def _ub(self, s, env) -> int:
        return int(s.ub) if isinstance(s.ub, int) else int(env[s.ub])

    def _stmt(self, s: Stmt, env):
        from . import device

        k = s.kind
        if k == "Stencil2DMVM":
            st = env[s.args[0]]
            w, ox, oy = st.taps()
            env[s.dst] = device.stencil2d(w, ox, oy, env[s.args[1]])
        elif k == "Array2DOp":
            env[s.dst] = device.array2d_op(L.OP_CODES[s.op], env[s.args[0]], env[s.args[1]])
        elif k == "Array2DScalarOp":
            env[s.dst] = device.array2d_scalar_op(L.OP_CODES[s.op], env[s.args[0]],
                                                  np.float32(env[s.args[1]]))
        elif k == "ScalarArray2DOp":
            env[s.dst] = device.scalar_array2d_op(L.OP_CODES[s.op], np.float32(env[s.args[0]]),
                                                  env[s.args[1]])
        elif k == "ScalarOp":
            a, b = np.float32(env[s.args[0]]), np.float32(env[s.args[1]])
            env[s.dst] = {"Add": a + b, "Sub": a - b, "Mult": a * b, "Div": _fdiv(a, b)}[s.op]
        elif k == "ScalarNeg":
            env[s.dst] = -np.float32(env[s.args[0]])
        elif k == "Const":
            env[s.dst] = s.args[0]
        elif k in ("Array2DCopy", "ScalarCopy", "Array3DCopy"):
            env[s.dst] = env[s.args[0]]  # values are never updated in place: rebinding is a copy
        elif k == "Fused":
            from .fusion import run_group, split_group

            fast = bool(self.defines.get("hs_fast_math", False))
            if not run_group(s, env, fast, self.stats):
                for part in split_group(s):
                    run_group(part, env, fast, self.stats)
        elif k in ("Array2DSqrt", "RedArray2D", "BlackArray2D", "Array2DSum"):
            # no stand-alone operator: a one-statement kernel (fusion switched off)
            from .fusion import run_group, split_group

            for part in split_group(Stmt("Fused", None, (), info={"stmts": [s], "id": 0})):
                run_group(part, env, bool(self.defines.get("hs_fast_math", False)), self.stats)
        elif k == "ScalarSqrt":
            env[s.dst] = np.sqrt(np.float32(env[s.args[0]]), dtype=np.float32)
        elif k == "WarpImg2D":
            env[s.dst] = device.warp(env[s.args[0]], env[s.args[1]], env[s.args[2]])
        elif k == "SpmvDIA2D":
            from .flow import spmv_dia2d

            env[s.dst] = spmv_dia2d(env[s.args[0]], env[s.args[1]])
        elif k == "SetBroxMatrix":
            from .flow import set_brox_matrix

            set_brox_matrix(env[s.args[0]], env[s.args[1]], np.float32(env[s.args[2]]))
        elif k == "SetBroxRedblackMatrix":
            from .flow import set_brox_redblack_matrix

            env[s.dst] = set_brox_redblack_matrix(env[s.args[0]], env[s.args[1]],
                                                  np.float32(env[s.args[2]]))
        elif k == "ApplyBroxPreconditioner":
            from .flow import apply_brox_preconditioner

            y0, y1 = apply_brox_preconditioner(*(env[a] for a in s.args))
            env[s.info["dsts"][0]], env[s.info["dsts"][1]] = y0, y1
        elif k == "LKLeastSquares":
            from .flow import lk_least_squares

            rad = int(self.defines.get("RADIUS", 0))
            if rad < 1:
                raise HMCompileError("lk_least_squares needs defines['RADIUS'] >= 1")
            du, dv = lk_least_squares(*(env[a] for a in s.args), rad)
            env[s.info["dsts"][0]], env[s.info["dsts"][1]] = du, dv
        elif k == "ApplyHSPreconditioner":
            from .cg import apply_hs_preconditioner

            y0, y1 = apply_hs_preconditioner(*(env[a] for a in s.args))
            env[s.info["dsts"][0]], env[s.info["dsts"][1]] = y0, y1
        elif k == "HSMatrixPowers":
            from .cg import hs_matrix_powers

            steps = int(self.defines.get("STEPS", 0))
            if steps < 1:
                raise HMCompileError("hs_matrix_powers needs defines['STEPS'] >= 1")
            lam = np.float32(env[s.args[0]])
            V0, V1 = hs_matrix_powers(float(lam), *(env[a] for a in s.args[1:]), steps)
            env[s.info["dsts"][0]], env[s.info["dsts"][1]] = V0, V1
        elif k == "Iterator":
            for _ in range(self._ub(s, env)):
                r = self._block(s.body, env)
                if r is not None:
                    return r
        elif k == "HSSweeps":
            self._hs_sweeps(s, env)
        elif k == "Return":
            return s.args, s.info.get("tuple", False)
        else:
            raise HMCompileError(f"internal: unknown statement {k}")
        return None

    def _hs_sweeps(self, s: Stmt, env) -> None:
        from . import device

        m = s.info
        weights = hs_average_weights(env[m["A"]])
        iters = self._ub(s, env)
        if weights is None:
            # the stencil is not the symmetric 3x3 average the fused kernel computes
            self.stats["unfused_loops"] += 1
            for _ in range(iters):
                self._block(s.body, env)
            return
        we, wc = weights
        Ix, Iy, It = device._same_layout(env[m["Ix"]], env[m["Iy"]], env[m["It"]])
        u = _fresh_copy(env[m["U"]], Ix)
        v = _fresh_copy(env[m["V"]], Ix)
        cfg = self.config()
        if cfg.sweeps_per_pass == 0 and self.defines.get("hs_autotune", True):
            # no depth in `defines`: the fastest (depth, segment, layout) for this shape and
            # form on this device, timed once per process and cached (autotune.py)
            from .autotune import best_sweep_config

            T, seg, layout = best_sweep_config(Ix.shape[0], Ix.shape[1], Ix.stride(0),
                                               fast_math=bool(cfg.fast_math))
            cfg.sweeps_per_pass, cfg.layout = T, layout
            if cfg.rows_per_segment == 0:
                cfg.rows_per_segment = seg
        cfg.avg_edge = float(we)
        cfg.avg_corner = float(wc)
        device.hs_sweeps(Ix, Iy, It, np.float32(env[m["alpha2"]]), iters, u, v, cfg)
        self.stats["hs_sweeps_calls"] += 1
        self.last_sweep_config = (cfg.sweeps_per_pass, cfg.rows_per_segment, cfg.layout,
                                  bool(cfg.fast_math))
        env[m["U"]] = u
        env[m["V"]] = v


def _span(t) -> tuple:
    """(device, first byte, one past the last byte) that tensor t may touch."""
    lo = t.data_ptr()
    n = sum((d - 1) * st for d, st in zip(t.shape, t.stride())) + 1 if t.numel() else 0
    return (str(t.device), lo, lo + n * t.element_size())


def _overlap(a: tuple, b: tuple) -> bool:
    """True when two spans of _span share a byte."""
    return a[0] == b[0] and a[1] < b[2] and b[1] < a[2]


def _fdiv(a, b):
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.float32(a / b)


def _fresh_copy(x, like):
    """A new plane with `like`'s row stride holding x (hs_sweeps updates in place)."""
    import torch

    H, W = like.shape
    p = torch.empty((H, like.stride(0)), dtype=torch.float32, device=like.device)[:, :W]
    p.copy_(x)
    return p


def function_source(fn) -> str:
    return textwrap.dedent(inspect.getsource(fn))
