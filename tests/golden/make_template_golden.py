"""Generate fixtures from the reference's own device templates, for the operators whose
device path has no matching CPU implementation in the reference.

    python tests/golden/make_template_golden.py <path of the reference checkout>

The reference emits each operator's per-element kernel text from C++: an ElementLevel's
compile() fills a CodeTemplate (lm.cpp:1174-1217: addLine appends a line, replace(NAME, v)
substitutes every "<NAME>" in the order the calls are made) with operand accesses that the
operand classes spell:
  Array2DOperand::getElement()        name[element_id0 + element_id1 * dim0]
  Array2DOperand::getElement(o0, o1)  name[element_id0 + element_id1 * dim0 + (o0) + (o1) * dim0]
  Array2DOperand::get(o0, o1)         name[(o0) + (o1) * dim0]          (Types/Array2D.cpp:285-368)
  Array3DOperand::get(o0, o1, o2)     name[(o0) + (o1) * dim0 + (o2) * dim0 * dim1]
                                                                      (Types/Array3D.cpp:290-341)
  ScalarOperand::getElement()         *name                            (Types/Scalar.cpp:109-121)
  StencilOperand::getData(d), getOffx(d), getOffy(d)
                                      name[d], name_offx[d], name_offy[d]  (Types/Stencil.cpp:126-143)
  SpMat2DOperand::getDataElement(d, o0, o1)
                      name[element_id0 + element_id1 * dim0 + d * dim0 * dim1 + o0 + o1 * dim0]
  SpMat2DOperand::getOffxElement(d), getOffyElement(d)
                                      name_offx[d], name_offy[d]        (Types/SpMat2D.cpp:204-230)
with dim0 the row length of the row-major arrays (the SetupLaunch functions swap dim0/dim1
when col_mjr is not "True").  Each launch covers every element, and every element of a
launch is independent.

This script reads those compile() functions from the reference's source files, makes the
same substitutions for each fixture's sizes, wraps each launch's element body in a loop over
all elements, runs the launches in the order the SetupLaunch function issues them, compiles
that with gcc (C's arithmetic as the template spells it, one IEEE rounding per operation: no
contraction, no fast math) and runs it on seeded inputs.  Nothing of the reference is copied
into the repository; the generated C lives in a temporary directory.

Fixtures (tests/golden/tmpl_*.npz; n = number of cases, per case i the arrays below):
  tmpl_lk.npz         LKLeastSquares (Operations/OpticalFlow/LKLeastSquares.cpp:39-91).  The
                      reference's NumPy lk_least_squares (hlib.py:86-118) is a different
                      algorithm ((2r+1)^2 window, float64), so it cannot pin the device path.
                      err_i, Ix_i, Iy_i, rad_i, du_i, dv_i
  tmpl_matrix_powers.npz
                      HSMatrixPowers (Operations/OpticalFlow/HSMatrixPowers.cpp:28-126: the
                      copy into plane 0, then one launch per step 1 .. STEPS-1); hlib has no
                      counterpart.  lam_i, Ix_i, Iy_i, r0_i, r1_i, steps_i, V0_i, V1_i
  tmpl_warp.npz       WarpImg2D (Operations/OpticalFlow/WarpImg2D.cpp:33-75) at fractional
                      offsets; hlib's warp_img2d agrees with it only at integer offsets.
                      src_i, ox_i, oy_i, out_i
  tmpl_stencil.npz    Stencil2DMVM (Operations/StructuredGrid/Stencil2DMVM.cpp:34-59).
                      w_i, offx_i, offy_i (taps), x_i, out_i
  tmpl_precond.npz    ApplyHSPreconditioner (ApplyHSPreconditioner.cpp:46-97), with pixels whose
                      determinant is exactly float(1e-15) (the template compares
                      fabs(det) > 1e-15 in double, and float(1e-15) lies above 1e-15).
                      s2_i, d0_i, d1_i, od_i, x0_i, x1_i, y0_i, y1_i
  tmpl_brox.npz       SetBroxMatrix and SetBroxRedblackMatrix on matrices that start from random
                      values (the templates write only the entries whose neighbour exists),
                      SpmvDIA2D on the 5-diagonal matrix, ApplyBroxPreconditioner
                      (ApplyBroxPreconditioner.cpp:46-75) with determinants at float(1e-4).
                      alpha; psi_i, A0_i (5 planes), A_i, R0_i (4 planes), R_i, adiag_i, x_i,
                      ax_i, d0_i, d1_i, od_i, x0_i, x1_i, y0_i, y1_i
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


# ---------------------------------------------------------------- template instantiation

def strip_comments(code: str) -> str:
    """C++ source without its // and /* */ comments (string literals kept intact: kernel text
    may itself hold "//")."""
    out, i, n = [], 0, len(code)
    while i < n:
        c = code[i]
        if c == '"':
            j = i + 1
            while code[j] != '"':
                j += 2 if code[j] == "\\" else 1
            out.append(code[i:j + 1])
            i = j + 1
        elif code.startswith("//", i):
            i = code.find("\n", i)
            i = n if i < 0 else i
        elif code.startswith("/*", i):
            i = code.index("*/", i) + 2
        else:
            out.append(c)
            i += 1
    return "".join(out)


def extract_template(src: str, method: str):
    """(lines, replacements) of `method` (e.g. "LKLeastSquaresElementLevel::compile"), the
    commented-out calls left out."""
    start = src.index("void " + method)
    end = src.index("ss << ct.getText()", start)
    body = strip_comments(src[start:end])
    lines = re.findall(r'ct\.addLine\("((?:[^"\\]|\\.)*)"\);', body)
    reps = [(m.group(1), m.group(2).strip())
            for m in re.finditer(r'ct\.replace\("(\w+)",\s*([^;]*)\);', body)]
    assert lines and reps, method
    # string escapes as the C++ compiler reads them (the templates use only \n)
    lines = [l.replace("\\n", "\n") for l in lines]
    return lines, reps


def access(operands, expr, dim0, dim1):
    """The access string an operand method call produces (see the module docstring)."""
    m = re.fullmatch(r'(\w+)->(getElement|get)\((.*)\)', expr)
    assert m, expr
    name, kind = operands[m.group(1)]
    args = re.findall(r'"([^"]*)"', m.group(3))
    elem = "element_id0 + element_id1 * {}".format(dim0)
    if kind == "a2" and m.group(2) == "getElement" and not args:
        return "{}[{}]".format(name, elem)
    if kind == "a2" and m.group(2) == "getElement" and len(args) == 2:
        return "{}[{} + ({}) + ({}) * {}]".format(name, elem, args[0], args[1], dim0)
    if kind == "a2" and m.group(2) == "get" and len(args) == 2:
        return "{}[({}) + ({}) * {}]".format(name, args[0], args[1], dim0)
    if kind == "a3" and m.group(2) == "get" and len(args) == 3:
        return "{}[({}) + ({}) * {} + ({}) * {}]".format(name, args[0], args[1], dim0, args[2],
                                                        dim0 * dim1)
    if kind == "s" and m.group(2) == "getElement" and not args:
        return "*" + name
    if kind == "a2" and m.group(2) == "get" and len(args) == 1:
        return "{}[{}]".format(name, args[0])
    raise ValueError(expr)


def access_ext(operands, expr, dim0, dim1):
    """access() plus the stencil and sparse-matrix operand methods."""
    m = re.fullmatch(r'(\w+)->(\w+)\((.*)\)', expr)
    assert m, expr
    name, kind = operands[m.group(1)]
    meth = m.group(2)
    args = re.findall(r'"([^"]*)"', m.group(3))
    if kind == "stencil":
        return {"getData": "{}[{}]", "getOffx": "{}_offx[{}]", "getOffy": "{}_offy[{}]"}[meth].format(
            name, args[0])
    if kind == "spmat":
        if meth == "getDataElement":
            return "{}[element_id0 + element_id1 * {} + {} * {} + {} + {} * {}]".format(
                name, dim0, args[0], dim0 * dim1, args[1], args[2], dim0)
        return {"getOffxElement": "{}_offx[{}]", "getOffyElement": "{}_offy[{}]"}[meth].format(
            name, args[0])
    return access(operands, expr, dim0, dim1)


def instantiate(template, operands, ints, dim0, dim1) -> str:
    lines, reps = template
    text = "\n".join(lines) + "\n"
    for name, expr in reps:
        value = str(ints[expr]) if expr in ints else access_ext(operands, expr, dim0, dim1)
        text = text.replace("<" + name + ">", value)
    assert not re.search(r"<[A-Za-z_]\w*>", text), text
    return text


C_PRELUDE = ("#include <math.h>\n"  # the reference's kernel prelude (lm.cpp:455-464)
             "#define MAX(a,b) (((a) > (b)) ? (a) : (b))\n"
             "#define MIN(a,b) (((a) < (b)) ? (a) : (b))\n")


def compile_launches(fname, params, bodies, W, H, tmp):
    """A C function running each element body over all W x H elements, in order.  params:
    names of float arrays, or "int:" + name for int arrays."""
    loops = "".join(
        "  for (int element_id1 = 0; element_id1 < %d; ++element_id1)\n"
        "  for (int element_id0 = 0; element_id0 < %d; ++element_id0) {\n%s  }\n" % (H, W, b)
        for b in bodies)
    sig = ", ".join(("int *" + p[4:]) if p.startswith("int:") else ("float *" + p) for p in params)
    path = os.path.join(tmp, "%s_%dx%d_%d" % (fname, H, W, len(os.listdir(tmp))))
    open(path + ".c", "w").write(C_PRELUDE + "void %s(%s)\n{\n%s}\n" % (fname, sig, loops))
    subprocess.run(["gcc", "-O1", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    path + ".c", "-o", path + ".so", "-lm"], check=True)
    fn = getattr(ctypes.CDLL(path + ".so"), fname)
    fn.argtypes = [np.ctypeslib.ndpointer(np.int32 if p.startswith("int:") else np.float32,
                                          flags="C_CONTIGUOUS") for p in params]
    fn.restype = None
    return fn


def read(ref_root, rel):
    return open(os.path.join(ref_root, *rel.split("/"))).read()


# ---------------------------------------------------------------- LKLeastSquares

LK_OPERANDS = {"errOperand": ("err", "a2"), "IxOperand": ("Ix", "a2"), "IyOperand": ("Iy", "a2"),
               "duOperand": ("du", "a2"), "dvOperand": ("dv", "a2")}
LK_CASES = [  # (H, W, rad, kind)
    (1, 1, 1, "normal"), (9, 9, 2, "normal"), (12, 15, 2, "normal"), (20, 9, 3, "normal"),
    (40, 70, 5, "normal"), (33, 129, 7, "normal"), (64, 64, 16, "normal"),
    (77, 45, 4, "normal"), (50, 60, 3, "flat_patch"), (24, 24, 1, "image_like"),
]


def lk_inputs(rng, H, W, kind):
    err, Ix, Iy = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(3))
    if kind == "flat_patch":  # a zero-gradient region: det == 0 there
        Ix[10:30, 20:45] = 0
        Iy[10:30, 20:45] = 0
    elif kind == "image_like":  # gradients of a periodic ramp: many equal windows
        y, x = np.mgrid[0:H, 0:W]
        Ix = (np.float32(0.25) + (x % 3 == 0) * np.float32(0.5)).astype(np.float32)
        Iy = (np.float32(0.125) * (y % 2)).astype(np.float32)
    return err, Ix, Iy


def make_lk(ref_root, tmp):
    t = extract_template(read(ref_root, "Operations/OpticalFlow/LKLeastSquares.cpp"),
                         "LKLeastSquaresElementLevel::compile")
    rng = np.random.default_rng(2718)
    out = {"n": np.int32(len(LK_CASES))}
    for i, (H, W, rad, kind) in enumerate(LK_CASES):
        err, Ix, Iy = lk_inputs(rng, H, W, kind)
        body = instantiate(t, LK_OPERANDS, {"dim0": W, "dim1": H, "rad": rad}, W, H)
        fn = compile_launches("lk_ref", ["err", "Ix", "Iy", "du", "dv"], [body], W, H, tmp)
        du = np.full((H, W), np.nan, np.float32)
        dv = np.full((H, W), np.nan, np.float32)
        fn(err, Ix, Iy, du, dv)
        assert not np.isnan(du).any() and not np.isnan(dv).any()
        out.update({f"err_{i}": err, f"Ix_{i}": Ix, f"Iy_{i}": Iy, f"rad_{i}": np.int32(rad),
                    f"du_{i}": du, f"dv_{i}": dv})
    return out


# ---------------------------------------------------------------- HSMatrixPowers

MP_OPERANDS = {"V0Operand": ("V0", "a3"), "V1Operand": ("V1", "a3"), "lamOperand": ("lam", "s"),
               "IxOperand": ("Ix", "a2"), "IyOperand": ("Iy", "a2"), "v0Operand": ("v0", "a2"),
               "v1Operand": ("v1", "a2")}
MP_CASES = [(1, 1, 3), (2, 3, 2), (7, 5, 4), (16, 16, 1), (37, 29, 5), (64, 96, 9), (33, 130, 3)]


def make_matrix_powers(ref_root, tmp):
    src = read(ref_root, "Operations/OpticalFlow/HSMatrixPowers.cpp")
    copy_t = extract_template(src, "Array2DArray3DCopyElementLevel::compile")
    step_t = extract_template(src, "HSMatrixPowersElementLevel::compile")
    rng = np.random.default_rng(1414)
    out = {"n": np.int32(len(MP_CASES))}
    for i, (H, W, steps) in enumerate(MP_CASES):
        Ix, Iy, r0, r1 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(4))
        lam = np.array([rng.uniform(0.1, 4.0)], np.float32)
        bodies = [instantiate(copy_t, MP_OPERANDS, {}, W, H)]
        bodies += [instantiate(step_t, MP_OPERANDS, {"step": s, "width": W, "height": H}, W, H)
                   for s in range(1, steps)]
        fn = compile_launches("mp_ref", ["V0", "V1", "lam", "Ix", "Iy", "v0", "v1"], bodies, W, H,
                              tmp)
        V0 = np.full((steps, H, W), np.nan, np.float32)
        V1 = np.full((steps, H, W), np.nan, np.float32)
        fn(V0, V1, lam, Ix, Iy, r0, r1)
        assert not np.isnan(V0).any() and not np.isnan(V1).any()
        out.update({f"lam_{i}": lam[0], f"Ix_{i}": Ix, f"Iy_{i}": Iy, f"r0_{i}": r0,
                    f"r1_{i}": r1, f"steps_{i}": np.int32(steps), f"V0_{i}": V0, f"V1_{i}": V1})
    return out


# ---------------------------------------------------------------- WarpImg2D

WARP_OPERANDS = {"dstOperand": ("dst", "a2"), "srcOperand": ("src", "a2"),
                 "offsetXOperand": ("offx", "a2"), "offsetYOperand": ("offy", "a2")}
WARP_CASES = [(1, 1, 0.5), (5, 7, 1.5), (24, 31, 3.0), (40, 64, 6.0), (63, 17, 0.25)]


def make_warp(ref_root, tmp):
    t = extract_template(read(ref_root, "Operations/OpticalFlow/WarpImg2D.cpp"),
                         "WarpImg2DElementLevel::compile")
    rng = np.random.default_rng(3141)
    out = {"n": np.int32(len(WARP_CASES))}
    for i, (H, W, amp) in enumerate(WARP_CASES):
        src = rng.standard_normal((H, W)).astype(np.float32)
        ox = (rng.uniform(-amp, amp, (H, W))).astype(np.float32)
        oy = (rng.uniform(-amp, amp, (H, W))).astype(np.float32)
        # integer, zero, negative-zero and just-below-integer offsets among the fractional ones
        ox.flat[::7] = np.round(ox.flat[::7])
        oy.flat[::5] = -0.0
        ox.flat[3::11] = np.float32(-1e-7)
        body = instantiate(t, WARP_OPERANDS, {"dim0": W, "dim1": H}, W, H)
        fn = compile_launches("warp_ref", ["dst", "src", "offx", "offy"], [body], W, H, tmp)
        dst = np.full((H, W), np.nan, np.float32)
        fn(dst, src, ox, oy)
        assert not np.isnan(dst).any()
        out.update({f"src_{i}": src, f"ox_{i}": ox, f"oy_{i}": oy, f"out_{i}": dst})
    return out


# ---------------------------------------------------------------- Stencil2DMVM

ST_OPERANDS = {"dstOperand": ("dst", "a2"), "stencilOperand": ("st", "stencil"),
               "srcOperand": ("src", "a2")}


def hs_average_taps():
    """The Horn-Schunck average in row-major tap order: corners 1/12, edges 1/6."""
    ox, oy, w = [], [], []
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dx or dy:
                ox.append(dx)
                oy.append(dy)
                w.append(1.0 / 12.0 if dx and dy else 1.0 / 6.0)
    return np.array(w, np.float32), np.array(ox, np.int32), np.array(oy, np.int32)


def stencil_cases(rng):
    avg = hs_average_taps()
    dx = (np.array([-0.25, 0.25, -0.25, 0.25], np.float32), np.array([0, 1, 0, 1], np.int32),
          np.array([0, 0, 1, 1], np.int32))
    yy, xx = np.mgrid[-2:3, -2:3]
    b = np.outer([1, 4, 6, 4, 1], [1, 4, 6, 4, 1]).astype(np.float32) / np.float32(256)
    binom = (b.ravel(), xx.ravel().astype(np.int32), yy.ravel().astype(np.int32))
    odd = (rng.standard_normal(6).astype(np.float32), np.array([-3, 0, 2, 5, -1, 1], np.int32),
           np.array([1, -4, 0, 2, 3, -2], np.int32))
    return [(1, 1, avg), (1, 7, avg), (7, 1, dx), (2, 2, avg), (13, 17, avg), (13, 17, binom),
            (40, 33, dx), (21, 30, odd)]


def make_stencil(ref_root, tmp):
    t = extract_template(read(ref_root, "Operations/StructuredGrid/Stencil2DMVM.cpp"),
                         "Stencil2DMVMElementLevel::compile")
    rng = np.random.default_rng(1618)
    cases = stencil_cases(rng)
    out = {"n": np.int32(len(cases))}
    for i, (H, W, (w, ox, oy)) in enumerate(cases):
        x = rng.standard_normal((H, W)).astype(np.float32)
        body = instantiate(t, ST_OPERANDS, {"width": W, "height": H, "ndiags": len(w)}, W, H)
        fn = compile_launches("st_ref", ["dst", "st", "int:st_offx", "int:st_offy", "src"], [body],
                              W, H, tmp)
        dst = np.full((H, W), np.nan, np.float32)
        fn(dst, w, ox, oy, x)
        out.update({f"w_{i}": w, f"offx_{i}": ox, f"offy_{i}": oy, f"x_{i}": x, f"out_{i}": dst})
    return out


# ---------------------------------------------------------------- ApplyHSPreconditioner

PC_OPERANDS = {"diagOperand0": ("d0", "a2"), "diagOperand1": ("d1", "a2"),
               "offdiagOperand": ("od", "a2"), "srcOperand0": ("x0", "a2"),
               "srcOperand1": ("x1", "a2"), "stencilOperand": ("st", "stencil"),
               "dstOperand0": ("y0", "a2"), "dstOperand1": ("y1", "a2")}


def make_precond(ref_root, tmp):
    t = extract_template(read(ref_root, "Operations/OpticalFlow/ApplyHSPreconditioner.cpp"),
                         "ApplyHSPreconditionerElementLevel::compile")
    rng = np.random.default_rng(1732)
    cases = [(1, 1, 0.3), (5, 9, 0.25), (24, 31, 1.0), (16, 16, 0.0), (33, 20, -0.5)]
    out = {"n": np.int32(len(cases))}
    for i, (H, W, s2) in enumerate(cases):
        d0, d1, od, x0, x1 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(5))
        if s2 == 0.0:  # determinants exactly at, just below and just above float(1e-15)
            e = np.float32(1e-15)
            d0[:] = 1
            od[:] = 0
            d1.flat[0::3] = e
            d1.flat[1::3] = np.nextafter(e, np.float32(0))
            d1.flat[2::3] = -e
        st = np.array([0, 0, s2, 0, 0], np.float32)
        body = instantiate(t, PC_OPERANDS, {"dim0": W, "dim1": H}, W, H)
        fn = compile_launches("pc_ref", ["d0", "d1", "od", "x0", "x1", "st", "y0", "y1"], [body],
                              W, H, tmp)
        y0 = np.full((H, W), np.nan, np.float32)
        y1 = np.full((H, W), np.nan, np.float32)
        fn(d0, d1, od, x0, x1, st, y0, y1)
        out.update({f"s2_{i}": np.float32(s2), f"d0_{i}": d0, f"d1_{i}": d1, f"od_{i}": od,
                    f"x0_{i}": x0, f"x1_{i}": x1, f"y0_{i}": y0, f"y1_{i}": y1})
    return out


# ---------------------------------------------------------------- Brox

BROX_SET = {"psiOperand": ("psi", "a2"), "spmatOperand": ("A", "spmat"),
            "alphaOperand": ("alpha", "s"), "AdiagOperand": ("adiag", "a2")}
BROX_SPMV = {"dstOperand": ("y", "a2"), "srcOperand1": ("A", "spmat"), "srcOperand2": ("x", "a2")}
BROX_PC = dict(PC_OPERANDS, stencilOperand=("A", "spmat"))
BROX_OFFX = np.array([0, -1, 0, 1, 0], np.int32)  # SetBroxMatrix's diagonal order
BROX_OFFY = np.array([-1, 0, 0, 0, 1], np.int32)


def make_brox(ref_root, tmp):
    def tmpl(rel, cls):
        return extract_template(read(ref_root, "Operations/" + rel), cls + "ElementLevel::compile")
    t_set = tmpl("OpticalFlow/SetBroxMatrix.cpp", "SetBroxMatrix")
    t_rb = tmpl("OpticalFlow/SetBroxRedblackMatrix.cpp", "SetBroxRedblackMatrix")
    t_mv = tmpl("SparseLinearAlgebra/SpmvDIA2D.cpp", "SpmvDIA2D")
    t_pc = tmpl("OpticalFlow/ApplyBroxPreconditioner.cpp", "ApplyBroxPreconditioner")
    rng = np.random.default_rng(2236)
    alpha = np.array([0.75], np.float32)
    cases = [(1, 1), (2, 3), (9, 7), (24, 31), (40, 33)]
    out = {"n": np.int32(len(cases)), "alpha": alpha[0]}
    for i, (H, W) in enumerate(cases):
        dims = {"dim0": W, "dim1": H, "ndiags": 5}
        psi = rng.uniform(0.05, 2.0, (H, W)).astype(np.float32)
        A0 = rng.standard_normal((5, H, W)).astype(np.float32)
        R0 = rng.standard_normal((4, H, W)).astype(np.float32)
        A, R = A0.copy(), R0.copy()
        adiag = np.full((H, W), np.nan, np.float32)
        compile_launches("set_ref", ["A", "psi", "alpha"],
                         [instantiate(t_set, BROX_SET, dims, W, H)], W, H, tmp)(A, psi, alpha)
        compile_launches("rb_ref", ["A", "adiag", "psi", "alpha"],
                         [instantiate(t_rb, BROX_SET, dims, W, H)], W, H, tmp)(R, adiag, psi, alpha)
        x = rng.standard_normal((H, W)).astype(np.float32)
        ax = np.full((H, W), np.nan, np.float32)
        compile_launches("mv_ref", ["y", "A", "int:A_offx", "int:A_offy", "x"],
                         [instantiate(t_mv, BROX_SPMV, dims, W, H)], W, H, tmp)(
            ax, A, BROX_OFFX, BROX_OFFY, x)
        d0, d1, od, x0, x1 = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(5))
        if H * W > 20:  # determinants at float(1e-4) (the template compares in double)
            mid = A[2]
            d0.flat[::4] = (np.float32(1) - mid.flat[::4])
            d1.flat[::4] = (np.float32(1e-4) - mid.flat[::4])
            od.flat[::4] = 0
        y0 = np.full((H, W), np.nan, np.float32)
        y1 = np.full((H, W), np.nan, np.float32)
        compile_launches("bpc_ref", ["d0", "d1", "od", "x0", "x1", "A", "y0", "y1"],
                         [instantiate(t_pc, BROX_PC, dims, W, H)], W, H, tmp)(
            d0, d1, od, x0, x1, A, y0, y1)
        for k, v in (("psi", psi), ("A0", A0), ("A", A), ("R0", R0), ("R", R), ("adiag", adiag),
                     ("x", x), ("ax", ax), ("d0", d0), ("d1", d1), ("od", od), ("x0", x0),
                     ("x1", x1), ("y0", y0), ("y1", y1)):
            out[f"{k}_{i}"] = v
    return out


def main(ref_root: str):
    with tempfile.TemporaryDirectory() as tmp:
        for fname, make in (("tmpl_lk.npz", make_lk), ("tmpl_matrix_powers.npz", make_matrix_powers),
                            ("tmpl_warp.npz", make_warp),
                            ("tmpl_stencil.npz", make_stencil),
                            ("tmpl_precond.npz", make_precond),
                            ("tmpl_brox.npz", make_brox)):
            out = make(ref_root, tmp)
            np.savez_compressed(os.path.join(HERE, fname), **out)
            print("wrote", fname, int(out["n"]), "cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
