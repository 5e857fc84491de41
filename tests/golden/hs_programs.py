"""Horn-Schunck programs written in the Hindemith surface.

The same function bodies run two ways:
  * undecorated, under the reference's own NumPy library (hlib.Stencil et al.), in
    make_golden.py -- that produces the golden fixtures;
  * decorated with hindemith_b200's @hm in the tests -- that is the drop-in under test.
"""


def hs_jacobi(I0, I1, Dx, Dy, Dt, A, alpha2, u, v, sweeps):
    # derivatives: three stencils per image, combined pointwise
    Ix = Dx * I0 + Dx * I1
    Iy = Dy * I0 + Dy * I1
    It = Dt * I1 - Dt * I0
    den = alpha2 + Ix * Ix + Iy * Iy
    for i in range(sweeps):
        ubar = A * u
        vbar = A * v
        t = (Ix * ubar + Iy * vbar + It) / den
        u = ubar - Ix * t
        v = vbar - Iy * t
    return u, v


def hs_jacobi_20(I0, I1, Dx, Dy, Dt, A, alpha, u, v):
    # the reference's form: integer-literal loop bound, alpha squared by a ScalarOp
    alpha2 = alpha * alpha
    Ix = Dx * I0 + Dx * I1
    Iy = Dy * I0 + Dy * I1
    It = Dt * I1 - Dt * I0
    den = alpha2 + Ix * Ix + Iy * Iy
    for i in range(20):
        ubar = A * u
        vbar = A * v
        t = (Ix * ubar + Iy * vbar + It) / den
        u = ubar - Ix * t
        v = vbar - Iy * t
    return u, v


def hs_jacobi_commuted(I0, I1, Dx, Dy, Dt, A, alpha2, u, v, sweeps):
    # operands commuted and temporaries renamed: still the fused Horn-Schunck loop
    Ix = Dx * I0 + Dx * I1
    Iy = Dy * I0 + Dy * I1
    It = Dt * I1 - Dt * I0
    den = Iy * Iy + (Ix * Ix + alpha2)
    for i in range(sweeps):
        a = A * u
        b = A * v
        r = It + (b * Iy + a * Ix)
        q = r / den
        u, v = a - q * Ix, b - Iy * q
    return u, v


def hs_jacobi_reassociated(I0, I1, Dx, Dy, Dt, A, alpha2, u, v, sweeps):
    # the residual summed in another association: not the fused kernel's rounding, so
    # this program must run statement by statement
    Ix = Dx * I0 + Dx * I1
    Iy = Dy * I0 + Dy * I1
    It = Dt * I1 - Dt * I0
    den = alpha2 + Ix * Ix + Iy * Iy
    for i in range(sweeps):
        ubar = A * u
        vbar = A * v
        t = (Ix * ubar + (Iy * vbar + It)) / den
        u = ubar - Ix * t
        v = vbar - Iy * t
    return u, v
