// hs_pyramid.cu -- the coarse-to-fine pieces around the Horn-Schunck solver and their
// adjoints: binomial blur + 2x decimation, 2x bilinear flow upsampling, and the bilinear
// backward warp of WarpImg2D (Operations/OpticalFlow/WarpImg2D.cpp:33-75).
//
// All are one-pass HBM-bound maps.  The adjoints of the blur and of the upsampling are
// gathers (each output sums the inputs whose forward footprint covers it, clamps folded
// in), so they are deterministic; the warp's adjoint with respect to the source image
// scatters along the flow, summed in 64-bit fixed point so that the result does not depend
// on the order of the atomics (deterministic too).
#include <algorithm>

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
    // Off the borders (every coarse index the pixel needs exists and no tap is clamped) the
    // weights are the bare binomial taps: an even fine index p gathers coarse p/2-1, p/2,
    // p/2+1 with (1, 6, 1)/16, an odd one (p-1)/2 and (p+1)/2 with (4, 4)/16.  The same fused
    // multiply-adds in the same order as the general loop below, so the same bits.
    if (x >= 2 && x + 2 <= 2 * Wo - 2 && y >= 2 && y + 2 <= 2 * Ho - 2) {
        const float b0 = kBin5[0], b1 = kBin5[1], b2 = kBin5[2];
        const int mx = x >> 1;
        auto row = [&](int oy) {
            const float *rp = dout + (size_t)oy * ldo;
            if (x & 1) return fmaf(b1, __ldg(rp + mx + 1), fmaf(b1, __ldg(rp + mx), 0.f));
            return fmaf(b0, __ldg(rp + mx + 1), fmaf(b2, __ldg(rp + mx), fmaf(b0, __ldg(rp + mx - 1), 0.f)));
        };
        const int my = y >> 1;
        float acc;
        if (y & 1) {
            acc = fmaf(b1, row(my), 0.f);
            acc = fmaf(b1, row(my + 1), acc);
        } else {
            acc = fmaf(b0, row(my - 1), 0.f);
            acc = fmaf(b2, row(my), acc);
            acc = fmaf(b0, row(my + 1), acc);
        }
        din[(size_t)y * ld + x] = acc;
        return;
    }
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
    // Off the borders (no clamped index on either side) coarse q collects fine 2q-1, 2q, 2q+1
    // and 2q+2 with weights 1/4, 3/4, 3/4, 1/4 along each axis: the general loop's fused
    // multiply-adds in its order, so the same bits.
    if (qx >= 1 && qx <= Wc - 2 && 2 * qx + 2 <= W - 1 && qy >= 1 && qy <= Hc - 2 &&
        2 * qy + 2 <= H - 1) {
        auto row = [&](int y) {
            const float *rp = df + (size_t)y * ld + 2 * qx;
            float r = fmaf(0.25f, __ldg(rp - 1), 0.f);
            r = fmaf(0.75f, __ldg(rp), r);
            r = fmaf(0.75f, __ldg(rp + 1), r);
            return fmaf(0.25f, __ldg(rp + 2), r);
        };
        float acc = fmaf(0.25f, row(2 * qy - 1), 0.f);
        acc = fmaf(0.75f, row(2 * qy), acc);
        acc = fmaf(0.75f, row(2 * qy + 1), acc);
        acc = fmaf(0.25f, row(2 * qy + 2), acc);
        dc[(size_t)qy * ldc + qx] = scale * acc;
        return;
    }
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
// keeps the source value.  The four accumulations follow C's (and OpenCL C's) typing of
// the template's expressions, evaluated left to right: a product stays float until a
// double operand (1.0 - frac) joins it, and an accumulation whose term is double rounds
// the double sum to the float output:
//   o  = float(0 + src00 * (1.0 - xf) * (1.0 - yf))          all double
//   o  = float(o + float(src10 * xf) * (1.0 - yf))           float product, then double
//   o  = float(o + src01 * (1.0 - xf) * yf)                  all double
//   o  = o + float(float(src11 * xf) * yf)                    all float
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
        // explicit roundings: no FMA contraction, products left to right
        const double xd = xfrac, yd = yfrac;
        const double nx = __dsub_rn(1.0, xd), ny = __dsub_rn(1.0, yd);
        o = 0.0f;
        o = (float)__dadd_rn(o, __dmul_rn(__dmul_rn(__ldg(src + b), nx), ny));
        o = (float)__dadd_rn(o, __dmul_rn((double)__fmul_rn(__ldg(src + b + 1), xfrac), ny));
        o = (float)__dadd_rn(o, __dmul_rn(__dmul_rn(__ldg(src + b + ld), nx), yd));
        o = __fadd_rn(o, __fmul_rn(__fmul_rn(__ldg(src + b + ld + 1), xfrac), yfrac));
    } else {
        o = __ldg(src + i);
    }
    dst[i] = o;
}

// Adjoint of warp_kernel given g = dL/ddst.  dL/dsrc is a scatter along the flow (a
// source pixel collects from every destination pixel whose footprint covers it).  To make
// the sums independent of the order the atomics land in, every contribution is converted
// to a 64-bit fixed-point integer with one power-of-two scale per launch and added with
// integer atomics (integer addition is associative); a last pass converts the sums back.
//
// The scale: with m = max |g| < 2^(e+1), a contribution is at most m, and a source pixel
// collects at most Nmax = min(H W, (2F + 3)^2) contributions, F = max(|u|, |v|) (a source
// pixel within F + 1 of the destination).  The scale 2^k, k = 61 - (e + 1) - ceil(log2
// Nmax), keeps every sum below 2^61 in magnitude; each contribution is rounded to a
// multiple of 2^-k, i.e. to about m 2^-(60 - log2 Nmax) (2^-50 m at F = 12).

// ws[0] = max |g| bits, ws[1] = max(|u|, |v|) bits (non-negative floats order like their
// bit patterns as unsigned integers)
__global__ void __launch_bounds__(256) warp_adjoint_scale_kernel(const float *__restrict__ g,
                                                                 const float *__restrict__ ou,
                                                                 const float *__restrict__ ov,
                                                                 int H, int W, int ld,
                                                                 unsigned *__restrict__ ws) {
    // blocks stride over rows, threads over a row's columns (no per-element division); the
    // maximum does not depend on the order
    unsigned mg = 0u, mf = 0u;
    for (int y = blockIdx.x; y < H; y += gridDim.x) {
        const size_t r = (size_t)y * ld;
        for (int x = threadIdx.x; x < W; x += blockDim.x) {
            mg = max(mg, __float_as_uint(fabsf(__ldg(g + r + x))));
            mf = max(mf, max(__float_as_uint(fabsf(__ldg(ou + r + x))), __float_as_uint(fabsf(__ldg(ov + r + x)))));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mg = max(mg, __shfl_xor_sync(0xffffffffu, mg, o));
        mf = max(mf, __shfl_xor_sync(0xffffffffu, mf, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(ws, mg);
        atomicMax(ws + 1, mf);
    }
}

// log2 of the fixed-point scale from the two maxima; false when g or the flow is not finite
__device__ __forceinline__ bool warp_adjoint_scale(const unsigned *ws, int H, int W, int &k) {
    const float m = __uint_as_float(ws[0]), F = __uint_as_float(ws[1]);
    if (!(m <= 3.0e38f) || !(F <= 3.0e38f)) return false;
    if (m == 0.f) {
        k = 0;
        return true;
    }
    const double side = 2.0 * ceil((double)F) + 3.0;
    const double nmax = fmin((double)H * (double)W, side * side);
    const int hb = (int)ceil(log2(fmax(nmax, 1.0)));
    k = 61 - (ilogbf(m) + 1) - hb;
    return true;
}

__global__ void __launch_bounds__(256) warp_adjoint_kernel(const float *__restrict__ src,
                                                           const float *__restrict__ ou,
                                                           const float *__restrict__ ov,
                                                           const float *__restrict__ g, int H,
                                                           int W, int ld,
                                                           const unsigned *__restrict__ scale,
                                                           unsigned long long *__restrict__ acc,
                                                           float *__restrict__ du,
                                                           float *__restrict__ dv) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    int k = 0;
    const bool finite = warp_adjoint_scale(scale, H, W, k);
    const size_t i = (size_t)y * ld + x;
    const float fx = __ldg(ou + i), fy = __ldg(ov + i), gi = __ldg(g + i);
    const int ix = (int)fx, iy = (int)fy;
    long long mx = ix, my = iy;
    float xf = __fsub_rn(fx, (float)ix), yf = __fsub_rn(fy, (float)iy);
    if (fx < 0.0f) { mx--; xf = (float)__dadd_rn(1.0, (double)xf); }
    if (fy < 0.0f) { my--; yf = (float)__dadd_rn(1.0, (double)yf); }
    // one contribution w * g as a fixed-point integer (two's complement wraps like the sum)
    auto add = [&](size_t q, double w) {
        if (!finite) return;
        const long long c = __double2ll_rn(scalbn(w * (double)gi, k));
        atomicAdd(acc + q, (unsigned long long)c);
    };
    if (x + mx >= 0 && x + mx + 1 < W && y + my >= 0 && y + my + 1 < H) {
        const size_t b = (size_t)(x + mx) + (size_t)(y + my) * ld;
        const float s00 = __ldg(src + b), s10 = __ldg(src + b + 1);
        const float s01 = __ldg(src + b + ld), s11 = __ldg(src + b + ld + 1);
        const double xd = xf, yd = yf, nx = 1.0 - xd, ny = 1.0 - yd;
        add(b, nx * ny);
        add(b + 1, xd * ny);
        add(b + ld, nx * yd);
        add(b + ld + 1, xd * yd);
        du[i] = gi * fmaf(yf, s11 - s01, (1.f - yf) * (s10 - s00));
        dv[i] = gi * fmaf(xf, s11 - s10, (1.f - xf) * (s01 - s00));
    } else {
        add(i, 1.0);
        du[i] = 0.f;
        dv[i] = 0.f;
    }
}

// dsrc = the fixed-point sums as floats (one rounding); NaN everywhere when g or the flow
// held a non-finite value
__global__ void __launch_bounds__(256) warp_adjoint_fold_kernel(const unsigned *__restrict__ scale,
                                                                const unsigned long long *__restrict__ acc,
                                                                int H, int W, int ld,
                                                                float *__restrict__ dsrc) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    int k = 0;
    const size_t i = (size_t)y * ld + x;
    if (!warp_adjoint_scale(scale, H, W, k)) {
        dsrc[i] = __int_as_float(0x7fc00000);
        return;
    }
    dsrc[i] = (float)scalbn((double)(long long)acc[i], -k);
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

size_t hs_warp_adjoint_workspace_bytes(int H, int W, int ld) {
    (void)W;
    if (H < 1 || ld < 1) return 0;
    return 256 + (sizeof(unsigned long long) * (size_t)H * (size_t)ld + 255) / 256 * 256;
}

hs_status hs_warp_adjoint(const float *src, const float *u, const float *v, const float *ddst,
                          int H, int W, int ld, float *dsrc, float *du, float *dv,
                          void *workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *pl[7] = {src, u, v, ddst, dsrc, du, dv};
    const char *nm[7] = {"src", "u", "v", "ddst", "dsrc", "du", "dv"};
    for (int k = 0; k < 7; ++k)
        if ((st = check_plane(pl[k], nm[k])) != HS_OK) return st;
    const size_t need = hs_warp_adjoint_workspace_bytes(H, W, ld);
    if (!workspace || workspace_bytes < need)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, need);
    if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
        HS_FAIL(HS_ERR_ALIGNMENT, "workspace is not 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned *scale = reinterpret_cast<unsigned *>(workspace);
    auto *acc = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(workspace) + 256);
    HS_CUDA_CHECK(cudaMemsetAsync(workspace, 0, need, s));
    const int blocks = std::min(H, sm_count() * 8);
    warp_adjoint_scale_kernel<<<std::max(blocks, 1), 256, 0, s>>>(ddst, u, v, H, W, ld, scale);
    HS_LAUNCH_CHECK("warp_adjoint_scale_kernel");
    warp_adjoint_kernel<<<g2(H, W), dim3(64, 4), 0, s>>>(src, u, v, ddst, H, W, ld, scale, acc, du, dv);
    HS_LAUNCH_CHECK("warp_adjoint_kernel");
    warp_adjoint_fold_kernel<<<g2(H, W), dim3(64, 4), 0, s>>>(scale, acc, H, W, ld, dsrc);
    HS_LAUNCH_CHECK("warp_adjoint_fold_kernel");
    return HS_OK;
}

}  // extern "C"
