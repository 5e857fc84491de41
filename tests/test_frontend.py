"""Host logic of the @hm front end: symbol kinds, statement lists, Horn-Schunck loop
recognition, error behaviour.  No device work."""
import inspect

import numpy as np
import pytest

import hs_programs
from hindemith_b200 import Stencil, hs_average_stencil, hs_derivative_stencils
from hindemith_b200.frontend import HMCompileError, parse, symbol_kind
from hindemith_b200.hlib import hs_average_weights

A2, ST, SC = "Array2D", "Stencil", "Scalar"
HS_PARAMS = dict(I0=A2, I1=A2, Dx=ST, Dy=ST, Dt=ST, A=ST, alpha2=SC, u=A2, v=A2, sweeps=SC)


def kinds(stmts):
    return [s.kind for s in stmts]


def test_symbol_kinds():
    assert symbol_kind(np.zeros((3, 4), np.float32)) == A2
    assert symbol_kind(hs_average_stencil()) == ST
    assert symbol_kind(np.float32(1.0)) == SC
    assert symbol_kind(np.int64(3)) == SC
    with pytest.raises(HMCompileError):
        symbol_kind(np.zeros(3))
    with pytest.raises(HMCompileError):
        symbol_kind("text")


def test_hs_loop_is_lowered():
    prog = parse(inspect.getsource(hs_programs.hs_jacobi), HS_PARAMS)
    k = kinds(prog.body)
    assert "HSSweeps" in k and "Iterator" not in k
    m = prog.body[k.index("HSSweeps")].info
    assert (m["U"], m["V"], m["A"], m["Ix"], m["Iy"], m["It"], m["den"], m["alpha2"]) == \
        ("u", "v", "A", "Ix", "Iy", "It", "den", "alpha2")
    assert prog.body[-1].kind == "Return" and prog.body[-1].args == ("u", "v")


def test_literal_bound_and_scalar_op():
    params = dict(HS_PARAMS)
    params.pop("sweeps")
    params.pop("alpha2")
    params["alpha"] = SC
    prog = parse(inspect.getsource(hs_programs.hs_jacobi_20), params)
    k = kinds(prog.body)
    assert k[0] == "ScalarOp"
    s = prog.body[k.index("HSSweeps")]
    assert s.ub == 20 and s.info["alpha2"] in ("alpha2", "_f0")  # the ScalarOp result


def test_commuted_program_is_lowered():
    prog = parse(inspect.getsource(hs_programs.hs_jacobi_commuted), HS_PARAMS)
    assert "HSSweeps" in kinds(prog.body)


def test_reassociated_program_runs_unfused():
    prog = parse(inspect.getsource(hs_programs.hs_jacobi_reassociated), HS_PARAMS)
    k = kinds(prog.body)
    assert "HSSweeps" not in k and "Iterator" in k


def test_loop_temporary_live_after_loop_blocks_lowering():
    src = '''
def f(Ix, Iy, It, A, alpha2, u, v):
    den = alpha2 + Ix * Ix + Iy * Iy
    for i in range(5):
        ubar = A * u
        vbar = A * v
        t = (Ix * ubar + Iy * vbar + It) / den
        u = ubar - Ix * t
        v = vbar - Iy * t
    return u, v, t
'''
    p = dict(Ix=A2, Iy=A2, It=A2, A=ST, alpha2=SC, u=A2, v=A2)
    assert "HSSweeps" not in kinds(parse(src, p).body)
    assert "HSSweeps" in kinds(parse(src.replace("return u, v, t", "return u, v"), p).body)


def test_unsupported_constructs_raise():
    p = dict(x=A2, A=ST, s=SC)
    with pytest.raises(HMCompileError):
        parse("def f(x, A, s):\n    return x ** s\n", p)
    with pytest.raises(HMCompileError):
        parse("def f(x, A, s):\n    y = A + x\n    return y\n", p)
    with pytest.raises(HMCompileError):
        parse("def f(x, A, s):\n    while s:\n        x = x\n    return x\n", p)
    with pytest.raises(HMCompileError):
        parse("def f(x, A, s):\n    return z\n", p)
    with pytest.raises(HMCompileError):
        parse("def f(x, A, s):\n    for i in range(1, 3):\n        x = x\n    return x\n", p)


def test_tuple_assignment_swaps():
    prog = parse("def f(a, b):\n    a, b = b, a\n    return a, b\n", dict(a=A2, b=A2))
    # every right-hand side is snapshotted before any target is rebound
    copies = [s for s in prog.body if s.kind == "Array2DCopy"]
    assert [c.dst for c in copies[:2]] == ["_f0", "_f1"]


def test_stencil_type_and_weights():
    A = hs_average_stencil()
    assert A.ndiags == 8 and A.dtype == np.float32
    we, wc = hs_average_weights(A)
    assert we == np.float32(1 / 6) and wc == np.float32(1 / 12)
    # with a zero centre tap in row-major order: still the fused form
    ox = [-1, 0, 1, -1, 0, 1, -1, 0, 1]
    oy = [-1, -1, -1, 0, 0, 0, 1, 1, 1]
    w = [1, 2, 1, 2, 0, 2, 1, 2, 1]
    assert hs_average_weights(Stencil(np.float32(w) / 12, ox, oy)) is not None
    w[4] = 3
    assert hs_average_weights(Stencil(np.float32(w) / 12, ox, oy)) is None
    # taps in another order: not the fused kernel's summation order
    assert hs_average_weights(Stencil(A.data[::-1], A.offx[::-1], A.offy[::-1])) is None
    with pytest.raises(ValueError):
        Stencil(np.zeros(3, np.float32), [0, 1], [0, 1, 2])
    dx, dy, dt = hs_derivative_stencils()
    assert dx.ndiags == dy.ndiags == dt.ndiags == 4


def test_fusion_groups_and_liveness():
    """Grouping follows the stencil-read vs element-write split rule, hoists host scalar
    statements, keeps dead intermediates out of the outputs and keeps loop-carried values."""
    from hindemith_b200.fusion import fuse_program

    src = '''
def f(x, y, A, a):
    p = A * x + y
    q = p * a + 1.0
    r = A * q
    for i in range(3):
        y = A * y + x
    return r, y
'''
    prog = parse(src, {"x": "Array2D", "y": "Array2D", "A": "Stencil", "a": "Scalar"})
    fuse_program(prog)
    kinds = [s.kind for s in prog.body]
    assert kinds.count("Fused") == 2 and "Iterator" in kinds
    g1, g2 = [s for s in prog.body if s.kind == "Fused"]
    # q is read by a stencil: the second group starts at `r = A * q`
    assert [t.kind for t in g2.info["stmts"]][0] == "Stencil2DMVM"
    assert "q" in g1.info["outputs"] and "p" not in g1.info["outputs"]
    # the Const 1.0 was hoisted in front of the first group
    assert prog.body.index(g1) > [s.kind for s in prog.body].index("Const")
    loop = next(s for s in prog.body if s.kind == "Iterator")
    (inner,) = [s for s in loop.body if s.kind == "Fused"]
    assert "y" in inner.info["outputs"]  # loop-carried


def test_fusion_codegen_body():
    from hindemith_b200.fusion import codegen, fuse_program
    from hindemith_b200 import hs_average_stencil

    src = '''
def f(x, A):
    m = sqrt(A * x + x)
    return m, sum2d(m)
'''
    prog = parse(src, {"x": "Array2D", "A": "Stencil"})
    fuse_program(prog)
    (g,) = [s for s in prog.body if s.kind == "Fused"]
    body, gen = codegen(g.info["stmts"], g.info["outputs"], g.info["sums"],
                        {"A": hs_average_stencil()})
    assert body.count("LD(0,") == 8 and "sqrtf(" in body and "SUM(0," in body and "OUT(0)" in body
    assert gen.inputs == ["x"]
    assert len(gen.scalars) == 2  # the two distinct weights of the average (1/6, 1/12)


def test_result_overlap_rule():
    """The rule that decides which results are copied: two tensors overlap when their byte
    spans on one device intersect (views of one plane do, neighbouring planes of one
    allocation do not)."""
    import torch

    from hindemith_b200.frontend import _overlap, _span

    buf = torch.empty((3, 5, 8), dtype=torch.float32)  # three padded 5 x 7 planes
    planes = [buf[i, :, :7] for i in range(3)]
    assert _overlap(_span(planes[0]), _span(planes[0]))
    assert _overlap(_span(planes[1]), _span(buf[1, 2:4, 3:5]))
    assert not _overlap(_span(planes[0]), _span(planes[1]))
    assert not _overlap(_span(planes[1]), _span(planes[2]))
    assert _overlap(_span(buf), _span(planes[2]))
    assert not _overlap(_span(torch.empty(0)), _span(planes[0]))
    other = torch.empty((5, 7))
    assert not _overlap(_span(other), _span(planes[0]))
    lo = _span(planes[0])
    assert not _overlap(("cuda:0",) + lo[1:], lo)  # same addresses on another device
