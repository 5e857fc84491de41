// hs_brox.cu -- the other flow methods on the same grid substrate: Lucas-Kanade least
// squares and the pieces of the Brox solver (its 5-diagonal smoothness matrix, the 2-D DIA
// product, the red-black variant and the 2x2 block preconditioner).  Each is one
// per-pixel kernel written in the reference templates' operation order (one rounding per
// operation), so results are bit-identical to their FP32 semantics.
#include <algorithm>

#include "hs_common.cuh"

namespace hs {

constexpr int kLkTile = 32;      // output tile edge
constexpr int kLkMaxRadius = 16;

// LKLeastSquares.cpp:44-79.  A 32 x 32 output tile per CTA (32 x 8 threads, 4 rows each);
// Ix, Iy and the error image are staged in shared memory with a halo of `rad` cells.
__global__ void __launch_bounds__(256) lk_kernel(const float *__restrict__ err,
                                                 const float *__restrict__ Ix,
                                                 const float *__restrict__ Iy, int H, int W,
                                                 int ld, int rad, float *__restrict__ du,
                                                 float *__restrict__ dv) {
    extern __shared__ float sm[];
    const int E = kLkTile + 2 * rad;
    float *sx = sm, *sy = sm + E * E, *se = sm + 2 * E * E;
    const int tx0 = blockIdx.x * kLkTile - rad, ty0 = blockIdx.y * kLkTile - rad;
    const int t = threadIdx.y * 32 + threadIdx.x;
    for (int c = t; c < E * E; c += 256) {
        const int x = tx0 + c % E, y = ty0 + c / E;
        float a = 0.f, b = 0.f, e = 0.f;
        if (x >= 0 && x < W && y >= 0 && y < H) {
            const size_t o = (size_t)y * ld + x;
            a = __ldg(Ix + o);
            b = __ldg(Iy + o);
            e = __ldg(err + o);
        }
        sx[c] = a;
        sy[c] = b;
        se[c] = e;
    }
    __syncthreads();
    const int x = blockIdx.x * kLkTile + threadIdx.x;
    for (int r = 0; r < 4; ++r) {
        const int y = blockIdx.y * kLkTile + threadIdx.y + 8 * r;
        if (x >= W || y >= H) continue;
        float u = 0.f, v = 0.f;
        if (x >= rad && y >= rad && x <= W - rad - 1 && y <= H - rad - 1) {
            float ix2 = 0.f, iy2 = 0.f, ixiy = 0.f, ixit = 0.f, iyit = 0.f;
            const int cx = x - tx0, cy = y - ty0;
            for (int dx = -rad; dx < rad; ++dx) {
                for (int dy = -rad; dy < rad; ++dy) {
                    const int c = (cy + dy) * E + (cx + dx);
                    const float a = sx[c], b = sy[c], e = se[c];
                    ix2 = __fadd_rn(ix2, __fmul_rn(a, a));
                    iy2 = __fadd_rn(iy2, __fmul_rn(b, b));
                    ixiy = __fadd_rn(ixiy, __fmul_rn(a, b));
                    ixit = __fadd_rn(ixit, __fmul_rn(a, e));
                    iyit = __fadd_rn(iyit, __fmul_rn(b, e));
                }
            }
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
    if (fabsf(det) > 1e-4f) {
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
    const int E = kLkTile + 2 * radius;
    const int smem = 3 * E * E * (int)sizeof(float);
    static bool attr[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(lk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           3 * (kLkTile + 2 * kLkMaxRadius) * (kLkTile + 2 * kLkMaxRadius) * (int)sizeof(float)));
        attr[dev] = true;
    }
    const dim3 grid((unsigned)((W + kLkTile - 1) / kLkTile), (unsigned)((H + kLkTile - 1) / kLkTile));
    lk_kernel<<<grid, dim3(32, 8), smem, (cudaStream_t)stream>>>(err, Ix, Iy, H, W, ld, radius, du, dv);
    HS_LAUNCH_CHECK("lk_kernel");
    return HS_OK;
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
