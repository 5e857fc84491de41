// hs_pyramid.cu -- the coarse-to-fine pieces around the Horn-Schunck solver and their
// adjoints: binomial blur + 2x decimation, 2x bilinear flow upsampling, and the bilinear
// backward warp of WarpImg2D (Operations/OpticalFlow/WarpImg2D.cpp:33-75).
//
// All are one-pass HBM-bound maps.  The adjoints of the blur and of the upsampling are
// gathers (each output sums the inputs whose forward footprint covers it, clamps folded
// in), so they are deterministic; the warp's adjoint with respect to the source image
// scatters along the flow with atomicAdd (float atomics: the summation order, hence the
// last bits, may vary between runs).
#include "hs_common.cuh"

namespace hs {

__constant__ float kBin5[5] = {1.f / 16, 4.f / 16, 6.f / 16, 4.f / 16, 1.f / 16};

// out[y][x] = sum_{dy,dx} b[dy] b[dx] in[clamp(2y+dy)][clamp(2x+dx)]
__global__ void __launch_bounds__(256) blur_down_kernel(const float *__restrict__ in, int H, int W,
                                                        int ld, float *__restrict__ out, int Ho,
                                                        int Wo, int ldo) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wo || y >= Ho) return;
    float acc = 0.f;
#pragma unroll
    for (int dy = -2; dy <= 2; ++dy) {
        const int yy = min(max(2 * y + dy, 0), H - 1);
        const float *row = in + (size_t)yy * ld;
        float r = 0.f;
#pragma unroll
        for (int dx = -2; dx <= 2; ++dx) r = fmaf(kBin5[dx + 2], __ldg(row + min(max(2 * x + dx, 0), W - 1)), r);
        acc = fmaf(kBin5[dy + 2], r, acc);
    }
    out[(size_t)y * ldo + x] = acc;
}

// Weight of coarse index o on fine index p along one axis: sum of b[d] over the taps d
// with clamp(2o + d, 0, n-1) == p.
__device__ __forceinline__ float down_weight(int o, int p, int n) {
    float w = 0.f;
#pragma unroll
    for (int d = -2; d <= 2; ++d) w += (min(max(2 * o + d, 0), n - 1) == p) ? kBin5[d + 2] : 0.f;
    return w;
}

// din[p] = sum over coarse o of w_y(o_y, p_y) w_x(o_x, p_x) dout[o]  (overwrites din)
__global__ void __launch_bounds__(256) blur_down_adjoint_kernel(const float *__restrict__ dout,
                                                                int Ho, int Wo, int ldo,
                                                                float *__restrict__ din, int H,
                                                                int W, int ld) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const int oy0 = max(0, (y - 3) / 2), oy1 = min(Ho - 1, (y + 3) / 2);
    const int ox0 = max(0, (x - 3) / 2), ox1 = min(Wo - 1, (x + 3) / 2);
    float acc = 0.f;
    for (int oy = oy0; oy <= oy1; ++oy) {
        const float wy = down_weight(oy, y, H);
        if (wy == 0.f) continue;
        float r = 0.f;
        for (int ox = ox0; ox <= ox1; ++ox) {
            const float wx = down_weight(ox, x, W);
            if (wx != 0.f) r = fmaf(wx, __ldg(dout + (size_t)oy * ldo + ox), r);
        }
        acc = fmaf(wy, r, acc);
    }
    din[(size_t)y * ld + x] = acc;
}

// 2x bilinear upsampling with half-pixel centres (coarse coordinate (i + 0.5)/2 - 0.5),
// coarse indices clamped; times `scale` (2 for flow, which doubles with the resolution).
__device__ __forceinline__ void up_axis(int i, int nc, int &i0, int &i1, float &f) {
    const float c = (i + 0.5f) * 0.5f - 0.5f;
    const float fl = floorf(c);
    f = c - fl;
    const int b = (int)fl;
    i0 = min(max(b, 0), nc - 1);
    i1 = min(max(b + 1, 0), nc - 1);
}

__global__ void __launch_bounds__(256) upsample2_kernel(const float *__restrict__ c, int Hc, int Wc,
                                                        int ldc, float *__restrict__ f, int H,
                                                        int W, int ld, float scale) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    int y0, y1, x0, x1;
    float fy, fx;
    up_axis(y, Hc, y0, y1, fy);
    up_axis(x, Wc, x0, x1, fx);
    const float *r0 = c + (size_t)y0 * ldc, *r1 = c + (size_t)y1 * ldc;
    const float top = fmaf(fx, __ldg(r0 + x1) - __ldg(r0 + x0), __ldg(r0 + x0));
    const float bot = fmaf(fx, __ldg(r1 + x1) - __ldg(r1 + x0), __ldg(r1 + x0));
    f[(size_t)y * ld + x] = scale * fmaf(fy, bot - top, top);
}

// dc[q] = scale * sum over fine p of w(p, q) df[p]  (overwrites dc)
__global__ void __launch_bounds__(256) upsample2_adjoint_kernel(const float *__restrict__ df, int H,
                                                                int W, int ld,
                                                                float *__restrict__ dc, int Hc,
                                                                int Wc, int ldc, float scale) {
    const int qx = blockIdx.x * blockDim.x + threadIdx.x;
    const int qy = blockIdx.y * blockDim.y + threadIdx.y;
    if (qx >= Wc || qy >= Hc) return;
    float acc = 0.f;
    for (int y = max(0, 2 * qy - 2); y <= min(H - 1, 2 * qy + 3); ++y) {
        int y0, y1;
        float fy;
        up_axis(y, Hc, y0, y1, fy);
        const float wy = (y0 == qy ? 1.f - fy : 0.f) + (y1 == qy ? fy : 0.f);
        if (wy == 0.f) continue;
        float r = 0.f;
        for (int x = max(0, 2 * qx - 2); x <= min(W - 1, 2 * qx + 3); ++x) {
            int x0, x1;
            float fx;
            up_axis(x, Wc, x0, x1, fx);
            const float wx = (x0 == qx ? 1.f - fx : 0.f) + (x1 == qx ? fx : 0.f);
            if (wx != 0.f) r = fmaf(wx, __ldg(df + (size_t)y * ld + x), r);
        }
        acc = fmaf(wy, r, acc);
    }
    // the coarse border also collects the clamped samples of fine pixels further out
    dc[(size_t)qy * ldc + qx] = scale * acc;
}

// WarpImg2D.cpp:33-75: the integer part truncates toward zero, then steps down for a
// negative offset; the fraction is a float; a pixel whose 2x2 footprint leaves the image
// keeps the source value.  As in the OpenCL template the weights are formed in double and
// each of the four accumulations rounds to the float output.
__global__ void __launch_bounds__(256) warp_kernel(const float *__restrict__ src,
                                                   const float *__restrict__ ou,
                                                   const float *__restrict__ ov, int H, int W,
                                                   int ld, float *__restrict__ dst) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * ld + x;
    const float fx = __ldg(ou + i), fy = __ldg(ov + i);
    // the conversion saturates for huge offsets; positions are formed in 64 bits so the
    // in-bounds test cannot overflow
    const int ix = (int)fx, iy = (int)fy;
    long long mx = ix, my = iy;
    float xfrac = __fsub_rn(fx, (float)ix), yfrac = __fsub_rn(fy, (float)iy);
    if (fx < 0.0f) { mx--; xfrac = (float)__dadd_rn(1.0, (double)xfrac); }
    if (fy < 0.0f) { my--; yfrac = (float)__dadd_rn(1.0, (double)yfrac); }
    float o;
    if (x + mx >= 0 && x + mx + 1 < W && y + my >= 0 && y + my + 1 < H) {
        const size_t b = (size_t)(x + mx) + (size_t)(y + my) * ld;
        // explicit roundings: no double FMA contraction, products left to right
        const double xd = xfrac, yd = yfrac;
        const double nx = __dsub_rn(1.0, xd), ny = __dsub_rn(1.0, yd);
        o = 0.0f;
        o = (float)__dadd_rn(o, __dmul_rn(__dmul_rn(__ldg(src + b), nx), ny));
        o = (float)__dadd_rn(o, __dmul_rn(__dmul_rn(__ldg(src + b + 1), xd), ny));
        o = (float)__dadd_rn(o, __dmul_rn(__dmul_rn(__ldg(src + b + ld), nx), yd));
        o = (float)__dadd_rn(o, __dmul_rn(__dmul_rn(__ldg(src + b + ld + 1), xd), yd));
    } else {
        o = __ldg(src + i);
    }
    dst[i] = o;
}

// Adjoint of warp_kernel given g = dL/ddst: dsrc += (scatter), du, dv (overwritten).
__global__ void __launch_bounds__(256) warp_adjoint_kernel(const float *__restrict__ src,
                                                           const float *__restrict__ ou,
                                                           const float *__restrict__ ov,
                                                           const float *__restrict__ g, int H,
                                                           int W, int ld,
                                                           float *__restrict__ dsrc,
                                                           float *__restrict__ du,
                                                           float *__restrict__ dv) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * ld + x;
    const float fx = __ldg(ou + i), fy = __ldg(ov + i), gi = __ldg(g + i);
    const int ix = (int)fx, iy = (int)fy;
    long long mx = ix, my = iy;
    float xf = __fsub_rn(fx, (float)ix), yf = __fsub_rn(fy, (float)iy);
    if (fx < 0.0f) { mx--; xf = (float)__dadd_rn(1.0, (double)xf); }
    if (fy < 0.0f) { my--; yf = (float)__dadd_rn(1.0, (double)yf); }
    if (x + mx >= 0 && x + mx + 1 < W && y + my >= 0 && y + my + 1 < H) {
        const size_t b = (size_t)(x + mx) + (size_t)(y + my) * ld;
        const float s00 = __ldg(src + b), s10 = __ldg(src + b + 1);
        const float s01 = __ldg(src + b + ld), s11 = __ldg(src + b + ld + 1);
        atomicAdd(dsrc + b, (1.f - xf) * (1.f - yf) * gi);
        atomicAdd(dsrc + b + 1, xf * (1.f - yf) * gi);
        atomicAdd(dsrc + b + ld, (1.f - xf) * yf * gi);
        atomicAdd(dsrc + b + ld + 1, xf * yf * gi);
        du[i] = gi * fmaf(yf, s11 - s01, (1.f - yf) * (s10 - s00));
        dv[i] = gi * fmaf(xf, s11 - s10, (1.f - xf) * (s01 - s00));
    } else {
        atomicAdd(dsrc + i, gi);
        du[i] = 0.f;
        dv[i] = 0.f;
    }
}

static inline dim3 g2(int H, int W) { return dim3((unsigned)((W + 63) / 64), (unsigned)((H + 3) / 4)); }

}  // namespace hs

using namespace hs;

extern "C" {

hs_status hs_blur_down(const float *in, int H, int W, int ld, float *out, int ldo, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const int Ho = (H + 1) / 2, Wo = (W + 1) / 2;
    if ((st = check_plane_geometry(Ho, Wo, ldo)) != HS_OK) return st;
    if ((st = check_plane(in, "in")) != HS_OK || (st = check_plane(out, "out")) != HS_OK) return st;
    blur_down_kernel<<<g2(Ho, Wo), dim3(64, 4), 0, (cudaStream_t)stream>>>(in, H, W, ld, out, Ho, Wo, ldo);
    HS_LAUNCH_CHECK("blur_down_kernel");
    return HS_OK;
}

hs_status hs_blur_down_adjoint(const float *dout, int H, int W, int ld, int ldo, float *din,
                               void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const int Ho = (H + 1) / 2, Wo = (W + 1) / 2;
    if ((st = check_plane_geometry(Ho, Wo, ldo)) != HS_OK) return st;
    if ((st = check_plane(dout, "dout")) != HS_OK || (st = check_plane(din, "din")) != HS_OK) return st;
    blur_down_adjoint_kernel<<<g2(H, W), dim3(64, 4), 0, (cudaStream_t)stream>>>(dout, Ho, Wo, ldo, din, H, W, ld);
    HS_LAUNCH_CHECK("blur_down_adjoint_kernel");
    return HS_OK;
}

hs_status hs_upsample2(const float *coarse, int ldc, float *fine, int H, int W, int ld,
                       float scale, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const int Hc = (H + 1) / 2, Wc = (W + 1) / 2;
    if ((st = check_plane_geometry(Hc, Wc, ldc)) != HS_OK) return st;
    if ((st = check_plane(coarse, "coarse")) != HS_OK || (st = check_plane(fine, "fine")) != HS_OK) return st;
    upsample2_kernel<<<g2(H, W), dim3(64, 4), 0, (cudaStream_t)stream>>>(coarse, Hc, Wc, ldc, fine, H, W, ld, scale);
    HS_LAUNCH_CHECK("upsample2_kernel");
    return HS_OK;
}

hs_status hs_upsample2_adjoint(const float *dfine, int H, int W, int ld, float *dcoarse, int ldc,
                               float scale, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const int Hc = (H + 1) / 2, Wc = (W + 1) / 2;
    if ((st = check_plane_geometry(Hc, Wc, ldc)) != HS_OK) return st;
    if ((st = check_plane(dfine, "dfine")) != HS_OK || (st = check_plane(dcoarse, "dcoarse")) != HS_OK) return st;
    upsample2_adjoint_kernel<<<g2(Hc, Wc), dim3(64, 4), 0, (cudaStream_t)stream>>>(dfine, H, W, ld, dcoarse, Hc, Wc, ldc, scale);
    HS_LAUNCH_CHECK("upsample2_adjoint_kernel");
    return HS_OK;
}

hs_status hs_warp(const float *src, const float *u, const float *v, int H, int W, int ld,
                  float *dst, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *pl[4] = {src, u, v, dst};
    const char *nm[4] = {"src", "u", "v", "dst"};
    for (int k = 0; k < 4; ++k)
        if ((st = check_plane(pl[k], nm[k])) != HS_OK) return st;
    if (src == dst) HS_FAIL(HS_ERR_INVALID_ARG, "src and dst must differ");
    warp_kernel<<<g2(H, W), dim3(64, 4), 0, (cudaStream_t)stream>>>(src, u, v, H, W, ld, dst);
    HS_LAUNCH_CHECK("warp_kernel");
    return HS_OK;
}

hs_status hs_warp_adjoint(const float *src, const float *u, const float *v, const float *ddst,
                          int H, int W, int ld, float *dsrc, float *du, float *dv, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *pl[7] = {src, u, v, ddst, dsrc, du, dv};
    const char *nm[7] = {"src", "u", "v", "ddst", "dsrc", "du", "dv"};
    for (int k = 0; k < 7; ++k)
        if ((st = check_plane(pl[k], nm[k])) != HS_OK) return st;
    warp_adjoint_kernel<<<g2(H, W), dim3(64, 4), 0, (cudaStream_t)stream>>>(src, u, v, ddst, H, W, ld, dsrc, du, dv);
    HS_LAUNCH_CHECK("warp_adjoint_kernel");
    return HS_OK;
}

}  // extern "C"
