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
with dim0 the row length of the row-major arrays (the SetupLaunch functions swap dim0/dim1
when col_mjr is not "True").  Each launch covers every element, and every element of a
launch is independent.

This script reads those compile() functions from the reference's source files, makes the
same substitutions for each fixture's sizes, wraps each launch's element body in a loop over
all elements, runs the launches in the order the SetupLaunch function issues them, compiles
that with gcc (C's arithmetic as the template spells it, one IEEE rounding per operation: no
contraction, no fast math) and runs it on seeded inputs.  Nothing of the reference is copied
into the repository; the generated C lives in a temporary directory.

Fixtures:
  lk.npz             LKLeastSquares (Operations/OpticalFlow/LKLeastSquares.cpp:39-91).  The
                     reference's NumPy lk_least_squares (hlib.py:86-118) is a different
                     algorithm ((2r+1)^2 window, float64), so it cannot pin the device path.
                     n; per case i: err_i, Ix_i, Iy_i, rad_i, du_i, dv_i
  matrix_powers.npz  HSMatrixPowers (Operations/OpticalFlow/HSMatrixPowers.cpp:28-126, the
                     copy into plane 0 then one launch per step 1 .. STEPS-1); hlib has no
                     counterpart.  n; per case i: lam_i, Ix_i, Iy_i, r0_i, r1_i, steps_i,
                     V0_i, V1_i (steps x H x W)
  warp_template.npz  WarpImg2D (Operations/OpticalFlow/WarpImg2D.cpp:33-75) at fractional
                     offsets; hlib's warp_img2d agrees with it only at integer offsets.
                     n; per case i: src_i, ox_i, oy_i, out_i
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

def extract_template(src: str, method: str):
    """(lines, replacements) of `method` (e.g. "LKLeastSquaresElementLevel::compile")."""
    start = src.index("void " + method)
    end = src.index("ss << ct.getText()", start)
    body = src[start:end]
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
    raise ValueError(expr)


def instantiate(template, operands, ints, dim0, dim1) -> str:
    lines, reps = template
    text = "\n".join(lines) + "\n"
    for name, expr in reps:
        value = str(ints[expr]) if expr in ints else access(operands, expr, dim0, dim1)
        text = text.replace("<" + name + ">", value)
    assert not re.search(r"<[A-Z][A-Z0-9]*>", text), text
    return text


def compile_launches(fname, params, bodies, W, H, tmp):
    """A C function running each element body over all W x H elements, in order."""
    loops = "".join(
        "  for (int element_id1 = 0; element_id1 < %d; ++element_id1)\n"
        "  for (int element_id0 = 0; element_id0 < %d; ++element_id0) {\n%s  }\n" % (H, W, b)
        for b in bodies)
    sig = ", ".join("float *" + p for p in params)
    path = os.path.join(tmp, "%s_%dx%d_%d" % (fname, H, W, len(os.listdir(tmp))))
    open(path + ".c", "w").write("void %s(%s)\n{\n%s}\n" % (fname, sig, loops))
    subprocess.run(["gcc", "-O1", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    path + ".c", "-o", path + ".so"], check=True)
    fn = getattr(ctypes.CDLL(path + ".so"), fname)
    fn.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")] * len(params)
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


def main(ref_root: str):
    with tempfile.TemporaryDirectory() as tmp:
        for fname, make in (("lk.npz", make_lk), ("matrix_powers.npz", make_matrix_powers),
                            ("warp_template.npz", make_warp)):
            out = make(ref_root, tmp)
            np.savez_compressed(os.path.join(HERE, fname), **out)
            print("wrote", fname, int(out["n"]), "cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
