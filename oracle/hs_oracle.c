/*
 * hs_oracle.c -- CPU restatement of the reference's Horn-Schunck stencil path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py call it through ctypes.  The
 * product (hindemith_b200 and libhsflow.so) never links or calls it.
 *
 * What it restates (file:line are paths inside chick/hindemith):
 *   - Stencil2DMVM element template, Operations/StructuredGrid/Stencil2DMVM.cpp:34-59:
 *       y = 0; for d < ndiags: x_ = clamp(x + offx[d], 0, W-1);
 *                              y_ = clamp(y + offy[d], 0, H-1);
 *                              y += S[d] * in[x_ + y_ * W]
 *     accumulated from 0 in tap order; index x + y*W (Types/Array2D.cpp:302,333).
 *   - Array2DOp / Array2DScalarOp / ScalarArray2DOp, a = b op c
 *     (Operations/DenseLinearAlgebra/Array2DOp.cpp:27-53, Array2DScalarOp.cpp:29-55,
 *      ScalarArray2DOp.cpp:29-55).
 *   - The Horn-Schunck program composed from those ops and fused the way
 *     fusion.cpp:113-303 fuses it: kernel A = both averages + the residual chain,
 *     storing ubar, vbar, t; kernel B = the write-back u, v.
 *   - WarpImg2D element template, Operations/OpticalFlow/WarpImg2D.cpp:33-75.
 *
 * The FP32 functions perform every operation in the reference program's order with
 * single rounding per operation (build with -ffp-contract=off), so they reproduce
 * the reference's FP32 semantics bit for bit.  The FP64 functions run the same
 * operator in double precision and serve as the accuracy reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HSO_API __attribute__((visibility("default")))

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Canonical Horn-Schunck stencils in tap order (offx, offy, weight).
 * Average: the 3x3 (1/12, 1/6) stencil without centre, row-major taps.
 * Derivatives: 2x2x2 first differences over the {0,1}^2 block, weight 1/4. */
static const int AVG_OX[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
static const int AVG_OY[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
static const int D_OX[4] = {0, 1, 0, 1};
static const int D_OY[4] = {0, 0, 1, 1};
static const float DX_W[4] = {-0.25f, 0.25f, -0.25f, 0.25f};
static const float DY_W[4] = {-0.25f, -0.25f, 0.25f, 0.25f};
static const float DT_W[4] = {0.25f, 0.25f, 0.25f, 0.25f};

static inline float avg_w_f32(int d) {
    /* corners 1/12, edges 1/6 */
    const float c = (float)(1.0 / 12.0), e = (float)(1.0 / 6.0);
    return (AVG_OX[d] != 0 && AVG_OY[d] != 0) ? c : e;
}

HSO_API int hso_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Threads of the following parallel loops (the timed CPU legs run at 1 and at all cores). */
HSO_API void hso_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---------------------------------------------------------------- stencils */

/* Stencil2DMVM.cpp:34-59, FP32, tap order. */
HSO_API void hso_stencil2d_f32(const float *w, const int *offx, const int *offy, int ntaps,
                               const float *in, float *out, int H, int W) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            float acc = 0.0f;
            for (int d = 0; d < ntaps; ++d) {
                int xx = clampi(x + offx[d], 0, W - 1);
                int yy = clampi(y + offy[d], 0, H - 1);
                float p = w[d] * in[xx + (size_t)yy * W];
                acc = acc + p;
            }
            out[x + (size_t)y * W] = acc;
        }
    }
}

HSO_API void hso_stencil2d_f64(const double *w, const int *offx, const int *offy, int ntaps,
                               const double *in, double *out, int H, int W) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            double acc = 0.0;
            for (int d = 0; d < ntaps; ++d) {
                int xx = clampi(x + offx[d], 0, W - 1);
                int yy = clampi(y + offy[d], 0, H - 1);
                acc += w[d] * in[xx + (size_t)yy * W];
            }
            out[x + (size_t)y * W] = acc;
        }
    }
}

/* Transposed clamp-to-edge stencil: out = S^T in, written as a gather.  Used by the
 * adjoint checks.  (S^T in)(p) = sum over q, d with clamp(q + off_d) == p of w_d in(q). */
HSO_API void hso_stencil2d_transpose_f64(const double *w, const int *offx, const int *offy,
                                         int ntaps, const double *in, double *out, int H, int W) {
    memset(out, 0, sizeof(double) * (size_t)H * W);
    /* scatter form, serial: exact and simple, used only at small sizes */
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int d = 0; d < ntaps; ++d) {
                int xx = clampi(x + offx[d], 0, W - 1);
                int yy = clampi(y + offy[d], 0, H - 1);
                out[xx + (size_t)yy * W] += w[d] * in[x + (size_t)y * W];
            }
}

/* ------------------------------------------------------------- derivatives */

/* Ix = Dx*I0 + Dx*I1; Iy = Dy*I0 + Dy*I1; It = Dt*I1 - Dt*I0 (Array2DOp Add/Sub of
 * Stencil2DMVM results), FP32 in program order. */
HSO_API void hso_hs_derivs_f32(const float *I0, const float *I1, int H, int W, float *Ix,
                               float *Iy, float *It) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            float ax0 = 0.f, ax1 = 0.f, ay0 = 0.f, ay1 = 0.f, at0 = 0.f, at1 = 0.f;
            for (int d = 0; d < 4; ++d) {
                int xx = clampi(x + D_OX[d], 0, W - 1);
                int yy = clampi(y + D_OY[d], 0, H - 1);
                float a = I0[xx + (size_t)yy * W], b = I1[xx + (size_t)yy * W];
                float p;
                p = DX_W[d] * a; ax0 = ax0 + p;
                p = DX_W[d] * b; ax1 = ax1 + p;
                p = DY_W[d] * a; ay0 = ay0 + p;
                p = DY_W[d] * b; ay1 = ay1 + p;
                p = DT_W[d] * a; at0 = at0 + p;
                p = DT_W[d] * b; at1 = at1 + p;
            }
            size_t i = x + (size_t)y * W;
            Ix[i] = ax0 + ax1;
            Iy[i] = ay0 + ay1;
            It[i] = at1 - at0;
        }
    }
}

HSO_API void hso_hs_derivs_f64(const double *I0, const double *I1, int H, int W, double *Ix,
                               double *Iy, double *It) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            double ax0 = 0, ax1 = 0, ay0 = 0, ay1 = 0, at0 = 0, at1 = 0;
            for (int d = 0; d < 4; ++d) {
                int xx = clampi(x + D_OX[d], 0, W - 1);
                int yy = clampi(y + D_OY[d], 0, H - 1);
                double a = I0[xx + (size_t)yy * W], b = I1[xx + (size_t)yy * W];
                ax0 += DX_W[d] * a; ax1 += DX_W[d] * b;
                ay0 += DY_W[d] * a; ay1 += DY_W[d] * b;
                at0 += DT_W[d] * a; at1 += DT_W[d] * b;
            }
            size_t i = x + (size_t)y * W;
            Ix[i] = ax0 + ax1;
            Iy[i] = ay0 + ay1;
            It[i] = at1 - at0;
        }
    }
}

/* ------------------------------------------------------------ Jacobi sweep */

/* Kernel A of the reference's fused sweep: ubar = A*u, vbar = A*v,
 * t = ((Ix*ubar + Iy*vbar) + It) / den with den = (alpha2 + Ix*Ix) + Iy*Iy. */
static void sweep_kernel_a_f32(const float *Ix, const float *Iy, const float *It, int H, int W,
                               float alpha2, const float *u, const float *v, float *ubar,
                               float *vbar, float *t) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            float au = 0.f, av = 0.f;
            for (int d = 0; d < 8; ++d) {
                int xx = clampi(x + AVG_OX[d], 0, W - 1);
                int yy = clampi(y + AVG_OY[d], 0, H - 1);
                float w = avg_w_f32(d);
                float p = w * u[xx + (size_t)yy * W];
                au = au + p;
                p = w * v[xx + (size_t)yy * W];
                av = av + p;
            }
            size_t i = x + (size_t)y * W;
            float ix = Ix[i], iy = Iy[i];
            float a = ix * au, b = iy * av;
            float r = a + b;
            r = r + It[i];
            float sq = ix * ix;
            float den = alpha2 + sq;
            sq = iy * iy;
            den = den + sq;
            ubar[i] = au;
            vbar[i] = av;
            t[i] = r / den;
        }
    }
}

/* Kernel B: u = ubar - Ix*t, v = vbar - Iy*t. */
static void sweep_kernel_b_f32(const float *Ix, const float *Iy, int n, const float *ubar,
                               const float *vbar, const float *t, float *u, float *v) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float p = Ix[i] * t[i];
        u[i] = ubar[i] - p;
        p = Iy[i] * t[i];
        v[i] = vbar[i] - p;
    }
}

/* `iters` Jacobi sweeps from the state in (u, v), in place. */
HSO_API int hso_hs_sweeps_f32(const float *Ix, const float *Iy, const float *It, int H, int W,
                              float alpha2, int iters, float *u, float *v) {
    size_t n = (size_t)H * W;
    float *ubar = (float *)malloc(sizeof(float) * n);
    float *vbar = (float *)malloc(sizeof(float) * n);
    float *t = (float *)malloc(sizeof(float) * n);
    if (!ubar || !vbar || !t) {
        free(ubar); free(vbar); free(t);
        return -1;
    }
    for (int k = 0; k < iters; ++k) {
        sweep_kernel_a_f32(Ix, Iy, It, H, W, alpha2, u, v, ubar, vbar, t);
        sweep_kernel_b_f32(Ix, Iy, (int)n, ubar, vbar, t, u, v);
    }
    free(ubar); free(vbar); free(t);
    return 0;
}

HSO_API int hso_hs_sweeps_f64(const double *Ix, const double *Iy, const double *It, int H, int W,
                              double alpha2, int iters, double *u, double *v) {
    size_t n = (size_t)H * W;
    double *ub = (double *)malloc(sizeof(double) * n);
    double *vb = (double *)malloc(sizeof(double) * n);
    if (!ub || !vb) { free(ub); free(vb); return -1; }
    for (int k = 0; k < iters; ++k) {
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y) {
            for (int x = 0; x < W; ++x) {
                double au = 0, av = 0;
                for (int d = 0; d < 8; ++d) {
                    int xx = clampi(x + AVG_OX[d], 0, W - 1);
                    int yy = clampi(y + AVG_OY[d], 0, H - 1);
                    double w = (double)avg_w_f32(d);
                    au += w * u[xx + (size_t)yy * W];
                    av += w * v[xx + (size_t)yy * W];
                }
                ub[x + (size_t)y * W] = au;
                vb[x + (size_t)y * W] = av;
            }
        }
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i) {
            double ix = Ix[i], iy = Iy[i];
            double den = alpha2 + ix * ix + iy * iy;
            double t = (ix * ub[i] + iy * vb[i] + It[i]) / den;
            u[i] = ub[i] - ix * t;
            v[i] = vb[i] - iy * t;
        }
    }
    free(ub); free(vb);
    return 0;
}

/* The whole plain path: derivatives, u = v = 0, `iters` sweeps.  alpha2 = alpha*alpha
 * (Horn & Schunck's convention: the smoothness weight enters the denominator squared). */
HSO_API int hso_hs_forward_f32(const float *I0, const float *I1, int H, int W, float alpha,
                               int iters, float *u, float *v) {
    size_t n = (size_t)H * W;
    float *Ix = (float *)malloc(sizeof(float) * n * 3);
    if (!Ix) return -1;
    float *Iy = Ix + n, *It = Iy + n;
    hso_hs_derivs_f32(I0, I1, H, W, Ix, Iy, It);
    memset(u, 0, sizeof(float) * n);
    memset(v, 0, sizeof(float) * n);
    float alpha2 = alpha * alpha;
    int rc = hso_hs_sweeps_f32(Ix, Iy, It, H, W, alpha2, iters, u, v);
    free(Ix);
    return rc;
}

HSO_API int hso_hs_forward_f64(const double *I0, const double *I1, int H, int W, double alpha,
                               int iters, double *u, double *v) {
    size_t n = (size_t)H * W;
    double *Ix = (double *)malloc(sizeof(double) * n * 3);
    if (!Ix) return -1;
    double *Iy = Ix + n, *It = Iy + n;
    hso_hs_derivs_f64(I0, I1, H, W, Ix, Iy, It);
    memset(u, 0, sizeof(double) * n);
    memset(v, 0, sizeof(double) * n);
    int rc = hso_hs_sweeps_f64(Ix, Iy, It, H, W, alpha * alpha, iters, u, v);
    free(Ix);
    return rc;
}

/* ------------------------------------------------------------------ warp */

/* WarpImg2D.cpp:33-75: backward bilinear warp of src by the offsets (ox, oy).  The
 * integer part truncates toward zero and is then floored for negative offsets; a
 * pixel whose 2x2 footprint leaves the image keeps the source value.  In OpenCL C, as
 * in C, the template's `1.0` literals are double and each expression is typed left to
 * right: `xfrac = 1.0 + xfrac` rounds back to the float variable; `IN * (1.0 - xfrac) *
 * (1.0 - yfrac)` is double throughout, `IN * (xfrac) * (1.0 - yfrac)` rounds the float
 * product IN * xfrac before the double one, and `IN * (xfrac) * (yfrac)` is all float;
 * `OUT += term` rounds a double sum to the float output, or adds in float for the float
 * term.  This restatement keeps exactly those roundings. */
HSO_API void hso_warp_f32(const float *src, const float *ox, const float *oy, int H, int W,
                          float *dst) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            size_t i = x + (size_t)y * W;
            float fx = ox[i], fy = oy[i];
            int mx = (int)fx, my = (int)fy;
            float xfrac = fx - (float)mx, yfrac = fy - (float)my;
            if (fx < 0.0) { mx--; xfrac = (float)(1.0 + (double)xfrac); }
            if (fy < 0.0) { my--; yfrac = (float)(1.0 + (double)yfrac); }
            if (x + mx >= 0 && x + mx + 1 < W && y + my >= 0 && y + my + 1 < H) {
                size_t b = (size_t)(x + mx) + (size_t)(y + my) * W;
                /* C's typing of the template's expressions, left to right: float products
                 * until (1.0 - frac) makes them double */
                float o = 0.0f;
                o = (float)((double)o + (double)src[b] * (1.0 - xfrac) * (1.0 - yfrac));
                o = (float)((double)o + (double)(src[b + 1] * xfrac) * (1.0 - yfrac));
                o = (float)((double)o + (double)src[b + W] * (1.0 - xfrac) * (double)yfrac);
                o = o + src[b + W + 1] * xfrac * yfrac;
                dst[i] = o;
            } else {
                dst[i] = src[i];
            }
        }
    }
}

/* ------------------------------------------------------------------ CG family */

/* HSMatrixPowers.cpp:72-106 (element template) and :129-226 (setup): V[0] = r; for
 * s = 1 .. steps-1, V[s] = M V[s-1] with the Horn-Schunck normal-equations operator
 *   ures = Ix*(Ix*u + Iy*v);  vres = Iy*(Ix*u + Iy*v)
 *   for each neighbour n present, in the order left (x > 0), right (x < W-1),
 *   up (y > 0), down (y < H-1):  res += -lam*n;  res += lam*mid
 * V is (steps, H, W), step slowest.  One rounding per operation, in template order. */
HSO_API void hso_hs_matrix_powers_f32(float lam, const float *Ix, const float *Iy, const float *r0,
                                      const float *r1, int H, int W, int steps, float *V0,
                                      float *V1) {
    const size_t n = (size_t)H * W;
    memcpy(V0, r0, n * sizeof(float));
    memcpy(V1, r1, n * sizeof(float));
    const float nl = -lam;
    for (int s = 1; s < steps; ++s) {
        const float *u = V0 + (size_t)(s - 1) * n, *v = V1 + (size_t)(s - 1) * n;
        float *uo = V0 + (size_t)s * n, *vo = V1 + (size_t)s * n;
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y) {
            for (int x = 0; x < W; ++x) {
                const size_t i = (size_t)y * W + x;
                const float um = u[i], vm = v[i], ix = Ix[i], iy = Iy[i];
                const float g = ix * um + iy * vm;
                float ur = ix * g, vr = iy * g;
                if (x > 0) { ur += nl * u[i - 1]; vr += nl * v[i - 1]; ur += lam * um; vr += lam * vm; }
                if (x < W - 1) { ur += nl * u[i + 1]; vr += nl * v[i + 1]; ur += lam * um; vr += lam * vm; }
                if (y > 0) { ur += nl * u[i - W]; vr += nl * v[i - W]; ur += lam * um; vr += lam * vm; }
                if (y < H - 1) { ur += nl * u[i + W]; vr += nl * v[i + W]; ur += lam * um; vr += lam * vm; }
                uo[i] = ur;
                vo[i] = vr;
            }
        }
    }
}

/* ApplyHSPreconditioner.cpp:46-97: the 2x2 block-Jacobi preconditioner of the HS system.
 *   a = diag0, d = diag1, each plus s for every neighbour present (x < W-1, y < H-1, x > 0,
 *   y > 0; s = the stencil's data[2]);  det = a*d - b*c (b = c = offdiag);
 *   |det| > 1e-15:  y0 = (x0*d - b*x1)/det,  y1 = (-c*x0 + a*x1)/det;  else y = x.
 * (hlib.applyHSPreconditioner, hlib.py:18-47, is the NumPy form; it tests |det| > 1e-4.) */
HSO_API void hso_apply_hs_precond_f32(float s2, const float *diag0, const float *diag1,
                                      const float *offdiag, const float *x0, const float *x1,
                                      int H, int W, float *y0, float *y1) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            float a = diag0[i], d = diag1[i];
            if (x < W - 1) { a += s2; d += s2; }
            if (y < H - 1) { a += s2; d += s2; }
            if (x > 0) { a += s2; d += s2; }
            if (y > 0) { a += s2; d += s2; }
            const float b = offdiag[i], c = offdiag[i], e = x0[i], f = x1[i];
            const float det = a * d - b * c;
            if ((double)fabsf(det) > 1e-15) { /* the template compares in double */
                y0[i] = (e * d - b * f) / det;
                y1[i] = (-c * e + a * f) / det;
            } else {
                y0[i] = e;
                y1[i] = f;
            }
        }
    }
}

/* ------------------------------------------------------------------ LK and Brox */

/* LKLeastSquares.cpp:44-79: per pixel at least `rad` from the left/top and rad+1 from the
 * right/bottom border, the 2x2 normal equations over the window dx, dy in [-rad, rad)
 * (dx outer, dy inner, float accumulation from 0), solved by Cramer's rule; 0 elsewhere
 * and where the determinant is 0. */
HSO_API void hso_lk_least_squares_f32(const float *err, const float *Ix, const float *Iy, int H,
                                      int W, int rad, float *du, float *dv) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            float u = 0.0f, v = 0.0f;
            if (x >= rad && y >= rad && x <= W - rad - 1 && y <= H - rad - 1) {
                float ix2 = 0.0f, iy2 = 0.0f, ixiy = 0.0f, ixit = 0.0f, iyit = 0.0f;
                for (int dx = -rad; dx < rad; ++dx) {
                    for (int dy = -rad; dy < rad; ++dy) {
                        const size_t j = (size_t)(y + dy) * W + (x + dx);
                        const float a = Ix[j], b = Iy[j], e = err[j];
                        ix2 += a * a;
                        iy2 += b * b;
                        ixiy += a * b;
                        ixit += a * e;
                        iyit += b * e;
                    }
                }
                const float det = ix2 * iy2 - ixiy * ixiy;
                if (det != 0.0f) {
                    u = (ixit * iy2 - ixiy * iyit) / det;
                    v = (ix2 * iyit - ixiy * ixit) / det;
                }
            }
            du[i] = u;
            dv[i] = v;
        }
    }
}

/* SetBroxMatrix.cpp:38-80 (redblack = 0: 5 diagonals top, left, mid, right, bottom) and
 * SetBroxRedblackMatrix.cpp:38-80 (redblack = 1: 4 diagonals top, left, right, bottom and
 * the mid term in adiag).  Diagonal d is a plane of the (ndiags, H, W) array `data`,
 * indexed by the column of the matrix entry (the neighbour): pixel (x, y) writes
 * top at (x, y-1), left at (x-1, y), right at (x+1, y), bottom at (x, y+1); entries no
 * pixel writes keep their values. */
HSO_API void hso_set_brox_matrix_f32(const float *psi, int H, int W, float alpha, float *data,
                                     int redblack, float *adiag) {
    const size_t P = (size_t)H * W;
    float *top = data, *left = data + P, *mid = redblack ? adiag : data + 2 * P;
    float *right = data + (redblack ? 2 : 3) * P, *bottom = data + (redblack ? 3 : 4) * P;
    const float na = -alpha;
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            float m = 0.0f;
            if (y > 0) { top[i - W] = na * psi[i - W]; m += alpha * psi[i - W]; }
            if (x > 0) { left[i - 1] = na * psi[i - 1]; m += alpha * psi[i - 1]; }
            if (x < W - 1) { right[i + 1] = na * psi[i]; m += alpha * psi[i]; }
            if (y < H - 1) { bottom[i + W] = na * psi[i]; m += alpha * psi[i]; }
            mid[i] = m;
        }
    }
}

/* SpmvDIA2D.cpp:36-45: y = 0; for each diagonal d with (x+offx, y+offy) inside the grid,
 * y += data[d][y+offy][x+offx] * x[y+offy][x+offx]. */
HSO_API void hso_spmv_dia2d_f32(const float *data, const int *offx, const int *offy, int ndiags,
                                const float *in, int H, int W, float *out) {
    const size_t P = (size_t)H * W;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            float acc = 0.0f;
            for (int d = 0; d < ndiags; ++d) {
                const int xx = x + offx[d], yy = y + offy[d];
                if (xx >= 0 && xx < W && yy >= 0 && yy < H) {
                    const size_t j = (size_t)yy * W + xx;
                    acc += data[d * P + j] * in[j];
                }
            }
            out[(size_t)y * W + x] = acc;
        }
    }
}

/* ApplyBroxPreconditioner.cpp:46-62: a = diag0 + mid, d = diag1 + mid (mid = the
 * matrix's middle diagonal at the pixel), det = a d - b c; |det| > 1e-4: the 2x2 solve,
 * else y = x. */
HSO_API void hso_apply_brox_precond_f32(const float *mid, const float *diag0, const float *diag1,
                                        const float *offdiag, const float *x0, const float *x1,
                                        int H, int W, float *y0, float *y1) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            const float a = diag0[i] + mid[i], d = diag1[i] + mid[i];
            const float b = offdiag[i], c = offdiag[i], e = x0[i], f = x1[i];
            const float det = a * d - b * c;
            if ((double)fabsf(det) > 1e-4) { /* the template compares in double */
                y0[i] = (e * d - b * f) / det;
                y1[i] = (-c * e + a * f) / det;
            } else {
                y0[i] = e;
                y1[i] = f;
            }
        }
    }
}
