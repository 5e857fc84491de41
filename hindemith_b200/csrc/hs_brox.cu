// hs_brox.cu -- the other flow methods on the same grid substrate: Lucas-Kanade least
// squares and the pieces of the Brox solver (its 5-diagonal smoothness matrix, the 2-D DIA
// product, the red-black variant and the 2x2 block preconditioner).  Each is one
// per-pixel kernel written in the reference templates' operation order (one rounding per
// operation), so results are bit-identical to their FP32 semantics.
#include <algorithm>

#include "hs_common.cuh"

namespace hs {

constexpr int kLkCols = 32;      // output columns per CTA (one per lane)
constexpr int kLkWarps = 4;      // warps per CTA, stacked vertically
constexpr int kLkMaxRadius = 16;

// The five products of one window cell c = (Ix, Iy, err, err), each rounded once:
// (Ix^2, Iy^2) and (Ix err, Iy err) as packed pairs, Ix Iy alone.
struct LkProd {
    float2 sq, et;
    float ab;
};
__device__ __forceinline__ LkProd lk_prod(float4 c) {
    const float2 xy = make_float2(c.x, c.y);
    return {mul2r(xy, xy), mul2r(xy, make_float2(c.z, c.w)), __fmul_rn(c.x, c.y)};
}

// LKLeastSquares.cpp:44-79.  Each pixel's five window sums run over dx in [-r, r) (outer)
// and dy in [-r, r) (inner), one rounding per operation, from 0.  A thread owns P
// vertically adjacent pixels of one column: it walks the cell columns dx and, in each, the
// P + 2r - 1 cell rows that the P windows cover, top to bottom, adding each cell's
// products to the pixels whose window holds that row.  Every pixel thus sees its cells in
// exactly the reference order, while a cell's products are formed once for up to P
// pixels.  The (Ix^2, Iy^2) and (Ix It, Iy It) sums are packed pairs.  Needs P - 1 <= 2r.
// The CTA stages its (32 + 2r) x (4P + 2r) cells as float4 (Ix, Iy, err, err) in shared
// memory; cells outside the image read 0 and feed only border pixels, whose flow is 0.
template <int P>
__global__ void __launch_bounds__(kLkCols * kLkWarps) lk_kernel(const float *__restrict__ err,
                                                                const float *__restrict__ Ix,
                                                                const float *__restrict__ Iy, int H,
                                                                int W, int ld, int rad,
                                                                float *__restrict__ du,
                                                                float *__restrict__ dv) {
    extern __shared__ float4 lk_cells[];
    const int ex = kLkCols + 2 * rad, ey = kLkWarps * P + 2 * rad;
    const int tx0 = blockIdx.x * kLkCols - rad, ty0 = blockIdx.y * (kLkWarps * P) - rad;
    const int t = threadIdx.y * kLkCols + threadIdx.x;
    for (int c = t; c < ex * ey; c += kLkCols * kLkWarps) {
        const int x = tx0 + c % ex, y = ty0 + c / ex;
        float a = 0.f, b = 0.f, e = 0.f;
        if (x >= 0 && x < W && y >= 0 && y < H) {
            const size_t o = (size_t)y * ld + x;
            a = __ldg(Ix + o);
            b = __ldg(Iy + o);
            e = __ldg(err + o);
        }
        lk_cells[c] = make_float4(a, b, e, e);
    }
    __syncthreads();

    const int lane = threadIdx.x, warp = threadIdx.y;
    float2 sq[P], et[P];
    float ab[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        sq[p] = et[p] = make_float2(0.f, 0.f);
        ab[p] = 0.f;
    }
    // pixel p (row warp*P + p of the CTA's outputs) has its window rows at cell rows
    // warp*P + p + [0, 2r) and its window columns at cell columns lane + [0, 2r)
    const float4 *col = lk_cells + (warp * P) * ex + lane;
    for (int dxi = 0; dxi < 2 * rad; ++dxi, ++col) {
#pragma unroll
        for (int j = 0; j < P - 1; ++j) {  // rows 0 .. P-2: pixels 0 .. j
            const LkProd q = lk_prod(col[j * ex]);
#pragma unroll
            for (int p = 0; p < P; ++p)
                if (p <= j) {
                    sq[p] = add2(sq[p], q.sq);
                    et[p] = add2(et[p], q.et);
                    ab[p] = __fadd_rn(ab[p], q.ab);
                }
        }
        for (int j = P - 1; j < 2 * rad; ++j) {  // rows P-1 .. 2r-1: every pixel
            const LkProd q = lk_prod(col[j * ex]);
#pragma unroll
            for (int p = 0; p < P; ++p) {
                sq[p] = add2(sq[p], q.sq);
                et[p] = add2(et[p], q.et);
                ab[p] = __fadd_rn(ab[p], q.ab);
            }
        }
#pragma unroll
        for (int k = 0; k < P - 1; ++k) {  // rows 2r .. 2r+P-2: pixels k+1 .. P-1
            const LkProd q = lk_prod(col[(2 * rad + k) * ex]);
#pragma unroll
            for (int p = 0; p < P; ++p)
                if (p > k) {
                    sq[p] = add2(sq[p], q.sq);
                    et[p] = add2(et[p], q.et);
                    ab[p] = __fadd_rn(ab[p], q.ab);
                }
        }
    }

    const int x = blockIdx.x * kLkCols + lane;
    if (x >= W) return;
    const bool xin = x >= rad && x <= W - rad - 1;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int y = blockIdx.y * (kLkWarps * P) + warp * P + p;
        if (y >= H) break;
        float u = 0.f, v = 0.f;
        if (xin && y >= rad && y <= H - rad - 1) {
            const float ix2 = sq[p].x, iy2 = sq[p].y, ixit = et[p].x, iyit = et[p].y, ixiy = ab[p];
            const float det = __fsub_rn(__fmul_rn(ix2, iy2), __fmul_rn(ixiy, ixiy));
            if (det != 0.f) {
                u = __fdiv_rn(__fsub_rn(__fmul_rn(ixit, iy2), __fmul_rn(ixiy, iyit)), det);
                v = __fdiv_rn(__fsub_rn(__fmul_rn(ix2, iyit), __fmul_rn(ixiy, ixit)), det);
            }
        }
        const size_t o = (size_t)y * ld + x;
        du[o] = u;
        dv[o] = v;
    }
}

template <int P>
hs_status launch_lk(const float *err, const float *Ix, const float *Iy, int H, int W, int ld,
                    int rad, float *du, float *dv, cudaStream_t s) {
    static bool attr[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        const int max_smem = (kLkCols + 2 * kLkMaxRadius) * (kLkWarps * P + 2 * kLkMaxRadius) * 16;
        HS_CUDA_CHECK(cudaFuncSetAttribute(lk_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
        attr[dev] = true;
    }
    const int smem = (kLkCols + 2 * rad) * (kLkWarps * P + 2 * rad) * 16;
    const dim3 grid((unsigned)((W + kLkCols - 1) / kLkCols), (unsigned)((H + kLkWarps * P - 1) / (kLkWarps * P)));
    lk_kernel<P><<<grid, dim3(kLkCols, kLkWarps), smem, s>>>(err, Ix, Iy, H, W, ld, rad, du, dv);
    HS_LAUNCH_CHECK("lk_kernel");
    return HS_OK;
}

// SetBroxMatrix.cpp:38-80 / SetBroxRedblackMatrix.cpp:38-80.  Each diagonal is indexed by
// the column of its matrix entry: pixel (x, y) writes top at (x, y-1), left at (x-1, y),
// right at (x+1, y) and bottom at (x, y+1), so every entry has at most one writer.
__global__ void __launch_bounds__(256) brox_set_kernel(const float *__restrict__ psi, int H, int W,
                                                       int ld, float alpha, float *top, float *left,
                                                       float *mid, float *right, float *bottom) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * ld + x;
    const float na = -alpha, p = __ldg(psi + i);
    float m = 0.f;
    if (y > 0) {
        const float q = __ldg(psi + i - ld);
        top[i - ld] = __fmul_rn(na, q);
        m = __fadd_rn(m, __fmul_rn(alpha, q));
    }
    if (x > 0) {
        const float q = __ldg(psi + i - 1);
        left[i - 1] = __fmul_rn(na, q);
        m = __fadd_rn(m, __fmul_rn(alpha, q));
    }
    if (x < W - 1) {
        right[i + 1] = __fmul_rn(na, p);
        m = __fadd_rn(m, __fmul_rn(alpha, p));
    }
    if (y < H - 1) {
        bottom[i + ld] = __fmul_rn(na, p);
        m = __fadd_rn(m, __fmul_rn(alpha, p));
    }
    mid[i] = m;
}

constexpr int kDiaMax = 16;
struct DiaOffsets {
    int offx[kDiaMax], offy[kDiaMax];
    int n;
};

// SpmvDIA2D.cpp:36-45.
__global__ void __launch_bounds__(256) spmv_dia2d_kernel(const float *__restrict__ data,
                                                         size_t dstride, const __grid_constant__ DiaOffsets o,
                                                         const float *__restrict__ in, int H, int W,
                                                         int ld, float *__restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float acc = 0.f;
    for (int d = 0; d < o.n; ++d) {
        const int xx = x + o.offx[d], yy = y + o.offy[d];
        if (xx >= 0 && xx < W && yy >= 0 && yy < H) {
            const size_t j = (size_t)yy * ld + xx;
            acc = __fadd_rn(acc, __fmul_rn(__ldg(data + d * dstride + j), __ldg(in + j)));
        }
    }
    out[(size_t)y * ld + x] = acc;
}

// ApplyBroxPreconditioner.cpp:46-62.
__global__ void __launch_bounds__(256) brox_precond_kernel(const float *__restrict__ mid,
                                                           const float *__restrict__ diag0,
                                                           const float *__restrict__ diag1,
                                                           const float *__restrict__ offdiag,
                                                           const float *__restrict__ x0,
                                                           const float *__restrict__ x1, int H,
                                                           int W, int ld, float *__restrict__ y0,
                                                           float *__restrict__ y1) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * ld + x;
    const float m = __ldg(mid + i);
    const float a = __fadd_rn(__ldg(diag0 + i), m), d = __fadd_rn(__ldg(diag1 + i), m);
    const float b = __ldg(offdiag + i), e = __ldg(x0 + i), f = __ldg(x1 + i);
    const float det = __fsub_rn(__fmul_rn(a, d), __fmul_rn(b, b));
    if ((double)fabsf(det) > 1e-4) {  // the template's double comparison
        y0[i] = __fdiv_rn(__fsub_rn(__fmul_rn(e, d), __fmul_rn(b, f)), det);
        y1[i] = __fdiv_rn(__fadd_rn(__fmul_rn(-b, e), __fmul_rn(a, f)), det);
    } else {
        y0[i] = e;
        y1[i] = f;
    }
}

static inline dim3 grid2(int H, int W) { return dim3((unsigned)((W + 63) / 64), (unsigned)((H + 3) / 4)); }

}  // namespace hs

using namespace hs;

extern "C" {

hs_status hs_lk_least_squares(const float *err, const float *Ix, const float *Iy, int H, int W,
                              int ld, int radius, float *du, float *dv, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *pl[5] = {err, Ix, Iy, du, dv};
    const char *nm[5] = {"err", "Ix", "Iy", "du", "dv"};
    for (int k = 0; k < 5; ++k)
        if ((st = check_plane(pl[k], nm[k])) != HS_OK) return st;
    if (radius < 1 || radius > kLkMaxRadius)
        HS_FAIL(HS_ERR_INVALID_ARG, "radius=%d outside 1..%d", radius, kLkMaxRadius);
    // pixels per thread: 8, or fewer where a window is shorter than 7 rows
    cudaStream_t s = (cudaStream_t)stream;
    if (radius >= 4) return launch_lk<8>(err, Ix, Iy, H, W, ld, radius, du, dv, s);
    if (radius >= 2) return launch_lk<4>(err, Ix, Iy, H, W, ld, radius, du, dv, s);
    return launch_lk<2>(err, Ix, Iy, H, W, ld, radius, du, dv, s);
}

hs_status hs_set_brox_matrix(const float *psi, int H, int W, int ld, float alpha, float *data,
                             size_t diag_stride, int redblack, float *adiag, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    if ((st = check_plane(psi, "psi")) != HS_OK || (st = check_plane(data, "data")) != HS_OK) return st;
    if (diag_stride < (size_t)H * ld || diag_stride % 4 != 0)
        HS_FAIL(HS_ERR_INVALID_ARG, "diag_stride=%zu must be >= H*ld and a multiple of 4", diag_stride);
    float *mid;
    if (redblack) {
        if ((st = check_plane(adiag, "adiag")) != HS_OK) return st;
        mid = adiag;
    } else {
        mid = data + 2 * diag_stride;
    }
    float *top = data, *left = data + diag_stride;
    float *right = data + (redblack ? 2 : 3) * diag_stride, *bottom = data + (redblack ? 3 : 4) * diag_stride;
    brox_set_kernel<<<grid2(H, W), dim3(64, 4), 0, (cudaStream_t)stream>>>(psi, H, W, ld, alpha, top, left,
                                                                             mid, right, bottom);
    HS_LAUNCH_CHECK("brox_set_kernel");
    return HS_OK;
}

hs_status hs_spmv_dia2d(const float *data, size_t diag_stride, const int *offx, const int *offy,
                        int ndiags, const float *x, int H, int W, int ld, float *y, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    if ((st = check_plane(data, "data")) != HS_OK || (st = check_plane(x, "x")) != HS_OK ||
        (st = check_plane(y, "y")) != HS_OK)
        return st;
    if (ndiags < 1 || ndiags > kDiaMax) HS_FAIL(HS_ERR_INVALID_ARG, "ndiags=%d outside 1..%d", ndiags, kDiaMax);
    if (!offx || !offy) HS_FAIL(HS_ERR_INVALID_ARG, "offx / offy are NULL");
    if (diag_stride < (size_t)H * ld || diag_stride % 4 != 0)
        HS_FAIL(HS_ERR_INVALID_ARG, "diag_stride=%zu must be >= H*ld and a multiple of 4", diag_stride);
    if (x == y) HS_FAIL(HS_ERR_INVALID_ARG, "x and y must differ");
    DiaOffsets o;
    memset(&o, 0, sizeof(o));
    o.n = ndiags;
    for (int d = 0; d < ndiags; ++d) {
        o.offx[d] = offx[d];
        o.offy[d] = offy[d];
    }
    spmv_dia2d_kernel<<<grid2(H, W), dim3(64, 4), 0, (cudaStream_t)stream>>>(data, diag_stride, o, x, H, W, ld, y);
    HS_LAUNCH_CHECK("spmv_dia2d_kernel");
    return HS_OK;
}

hs_status hs_apply_brox_preconditioner(const float *mid, const float *diag0, const float *diag1,
                                       const float *offdiag, const float *x0, const float *x1,
                                       int H, int W, int ld, float *y0, float *y1, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *pl[8] = {mid, diag0, diag1, offdiag, x0, x1, y0, y1};
    const char *nm[8] = {"mid", "diag0", "diag1", "offdiag", "x0", "x1", "y0", "y1"};
    for (int k = 0; k < 8; ++k)
        if ((st = check_plane(pl[k], nm[k])) != HS_OK) return st;
    brox_precond_kernel<<<grid2(H, W), dim3(64, 4), 0, (cudaStream_t)stream>>>(mid, diag0, diag1, offdiag,
                                                                                 x0, x1, H, W, ld, y0, y1);
    HS_LAUNCH_CHECK("brox_precond_kernel");
    return HS_OK;
}

}  // extern "C"
