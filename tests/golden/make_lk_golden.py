"""Generate tests/golden/lk.npz from the reference's own LKLeastSquares device template.

    python tests/golden/make_lk_golden.py <path of the reference checkout>

The reference computes Lucas-Kanade only on the device: LKLeastSquaresElementLevel::compile
(Operations/OpticalFlow/LKLeastSquares.cpp:39-91) emits the per-element kernel text through
a CodeTemplate (lm.cpp:1174-1217: addLine appends a line, replace(NAME, value) substitutes
every "<NAME>"), with operand accesses spelled by Array2DOperand::getElement
(Types/Array2D.cpp:297-368: "name[element_id0 + element_id1 * dim0 + (o0) + (o1) * dim0]").
Its NumPy lk_least_squares (hlib.py:86-118) is a different algorithm (a (2r+1)^2 window and
FP64), so it cannot pin the device path.

This script reads the template from the reference's source file, performs the same
substitutions for each fixture's dimensions and radius, wraps the resulting element body in
a C loop over every element (the launch covers all of them, each independent), compiles it
with gcc (one IEEE rounding per operation: no contraction, no fast math, as the other
fixtures' NumPy evaluation) and runs it on seeded inputs.  Nothing of the reference is
copied into the repository; the generated C lives in a temporary directory.

Fixture lk.npz: n, and per case i: err_i, Ix_i, Iy_i (H x W float32), rad_i, du_i, dv_i.
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

# Operand objects of LKLeastSquaresSetupLaunch -> the arrays they bind (LKLeastSquares.cpp:140-144)
OPERANDS = {"errOperand": "err", "IxOperand": "Ix", "IyOperand": "Iy",
            "duOperand": "du", "dvOperand": "dv"}

CASES = [  # (H, W, rad, kind)
    (1, 1, 1, "normal"), (9, 9, 2, "normal"), (12, 15, 2, "normal"), (20, 9, 3, "normal"),
    (40, 70, 5, "normal"), (33, 129, 7, "normal"), (64, 64, 16, "normal"),
    (77, 45, 4, "normal"), (50, 60, 3, "flat_patch"), (24, 24, 1, "image_like"),
]


def extract_template(src: str):
    """(lines, replacements) of LKLeastSquaresElementLevel::compile, in source order."""
    start = src.index("void LKLeastSquaresElementLevel::compile")
    end = src.index("ss << ct.getText()", start)
    body = src[start:end]
    lines = re.findall(r'ct\.addLine\("((?:[^"\\]|\\.)*)"\);', body)
    reps = []
    for m in re.finditer(r'ct\.replace\("(\w+)",\s*([^;]*)\);', body):
        reps.append((m.group(1), m.group(2).strip()))
    assert lines and reps, "template not found"
    return lines, reps


def instantiate(lines, reps, W: int, H: int, rad: int) -> str:
    """The element body with every <NAME> substituted as CodeTemplate::replace does."""
    dim0, dim1 = W, H  # row-major arrays: dim[0] = columns, dim[1] = rows
    text = "\n".join(lines) + "\n"
    elem = "element_id0 + element_id1 * {}".format(dim0)
    for name, expr in reps:
        m = re.fullmatch(r'(\w+)->getElement\(\)', expr)
        m2 = re.fullmatch(r'(\w+)->getElement\("(\w+)",\s*"(\w+)"\)', expr)
        if m:
            value = "{}[{}]".format(OPERANDS[m.group(1)], elem)
        elif m2:
            value = "{}[{} + ({}) + ({}) * {}]".format(OPERANDS[m2.group(1)], elem, m2.group(2),
                                                       m2.group(3), dim0)
        else:
            value = str({"dim0": dim0, "dim1": dim1, "rad": rad}[expr])
        text = text.replace("<" + name + ">", value)
    assert "<" not in text.replace("<=", "").replace(" < ", ""), text
    return text


def build_case(lines, reps, W, H, rad, tmp):
    body = instantiate(lines, reps, W, H, rad)
    c = ("void lk_ref(const float *err, const float *Ix, const float *Iy, float *du, float *dv)\n"
         "{\n  for (int element_id1 = 0; element_id1 < %d; ++element_id1)\n"
         "  for (int element_id0 = 0; element_id0 < %d; ++element_id0) {\n%s  }\n}\n"
         % (H, W, body))
    path = os.path.join(tmp, "lk_%dx%d_r%d" % (H, W, rad))
    open(path + ".c", "w").write(c)
    subprocess.run(["gcc", "-O1", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    path + ".c", "-o", path + ".so"], check=True)
    lib = ctypes.CDLL(path + ".so")
    fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    lib.lk_ref.argtypes = [fp] * 5
    lib.lk_ref.restype = None
    return lib.lk_ref


def inputs(rng, H, W, kind):
    err, Ix, Iy = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(3))
    if kind == "flat_patch":  # a zero-gradient region: det == 0 there
        Ix[10:30, 20:45] = 0
        Iy[10:30, 20:45] = 0
    elif kind == "image_like":  # gradients of a smooth ramp: many equal windows
        y, x = np.mgrid[0:H, 0:W].astype(np.float32)
        Ix = np.float32(0.25) * np.ones((H, W), np.float32) + (x % 3 == 0) * np.float32(0.5)
        Iy = np.float32(0.125) * (y % 2).astype(np.float32)
    return err, Ix, Iy


def main(ref_root: str):
    src = open(os.path.join(ref_root, "Operations", "OpticalFlow", "LKLeastSquares.cpp")).read()
    lines, reps = extract_template(src)
    rng = np.random.default_rng(2718)
    out = {"n": np.int32(len(CASES))}
    with tempfile.TemporaryDirectory() as tmp:
        for i, (H, W, rad, kind) in enumerate(CASES):
            err, Ix, Iy = inputs(rng, H, W, kind)
            fn = build_case(lines, reps, W, H, rad, tmp)
            du = np.full((H, W), np.nan, np.float32)
            dv = np.full((H, W), np.nan, np.float32)
            fn(err, Ix, Iy, du, dv)
            assert not np.isnan(du).any() and not np.isnan(dv).any()
            out.update({f"err_{i}": err, f"Ix_{i}": Ix, f"Iy_{i}": Iy, f"rad_{i}": np.int32(rad),
                        f"du_{i}": du, f"dv_{i}": dv})
    np.savez_compressed(os.path.join(HERE, "lk.npz"), **out)
    print("wrote", os.path.join(HERE, "lk.npz"), len(CASES), "cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
