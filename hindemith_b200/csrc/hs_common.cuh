// hs_common.cuh -- shared helpers of libhsflow: status plumbing, argument checks,
// launch helpers and the canonical Horn-Schunck stencil tables.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>

#include "../../include/hsflow.h"

namespace hs {

// Thread-local one-line detail of the last failing call (hs_last_error()).
void set_error(const char *fmt, ...);
void clear_error();

#define HS_FAIL(code, ...)               \
    do {                                 \
        ::hs::set_error(__VA_ARGS__);    \
        return (code);                   \
    } while (0)

#define HS_CUDA_CHECK(expr)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            HS_FAIL(HS_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));        \
    } while (0)

// Check the result of the kernel launch just issued.
#define HS_LAUNCH_CHECK(what)                                                            \
    do {                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess)                                                           \
            HS_FAIL(HS_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e_)); \
    } while (0)

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Plane geometry checks shared by every entry point.
inline hs_status check_plane_geometry(int H, int W, int ld) {
    if (H < 1 || W < 1) HS_FAIL(HS_ERR_INVALID_ARG, "H=%d W=%d must be >= 1", H, W);
    if (ld < W) HS_FAIL(HS_ERR_INVALID_ARG, "ld=%d < W=%d", ld, W);
    if (ld % 4 != 0) HS_FAIL(HS_ERR_ALIGNMENT, "ld=%d is not a multiple of 4 floats", ld);
    if ((long long)H * ld > (1LL << 40)) HS_FAIL(HS_ERR_INVALID_ARG, "plane too large");
    return HS_OK;
}

inline hs_status check_plane(const void *p, const char *name) {
    if (!p) HS_FAIL(HS_ERR_INVALID_ARG, "%s is NULL", name);
    if (!aligned16(p)) HS_FAIL(HS_ERR_ALIGNMENT, "%s is not 16-byte aligned", name);
    return HS_OK;
}

inline size_t plane_bytes(int H, int ld) { return sizeof(float) * (size_t)H * (size_t)ld; }

// Number of SMs of the current device (cached per device).
int sm_count();

// Canonical Horn-Schunck stencils.  Average: 3x3 without centre, corners 1/12, edges 1/6,
// taps row-major (dy = -1, 0, +1; dx = -1, 0, +1).  Derivatives: taps (0,0) (1,0) (0,1) (1,1).
constexpr float kAvgCorner = (float)(1.0 / 12.0);
constexpr float kAvgEdge = (float)(1.0 / 6.0);

#ifdef __CUDACC__
// Packed FP32 pairs (sm_100 f32x2 instructions: one instruction, two IEEE operations, each
// rounded to nearest even as its scalar form).
//   add2 / fma2: packed add and fused multiply-add.
//   mul2       : packed product, only where it feeds no add: the code generator fuses a
//                packed product into a following packed add (an FMA, which skips the
//                product's rounding) even with explicit .rn;
//   mul2r      : the product rounded on its own, as two scalar multiplies (never fused),
//                for the exact operation order.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
        "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "add.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
        "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mul.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 mul2r(float2 a, float2 b) {
    return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Horn-Schunck 2x2x2 derivatives at (x, y).  Tap order (0,0) (1,0) (0,1) (1,1), taps
// clamped to the image; each accumulator sums from 0 in that order, one rounding per
// operation; then Ix = DxI0 + DxI1, Iy = DyI0 + DyI1, It = DtI1 - DtI0.
__device__ __forceinline__ void hs_derivs_at(const float *__restrict__ I0,
                                             const float *__restrict__ I1, int x, int y, int H,
                                             int W, int ld, float &Ix, float &Iy, float &It) {
    const int x1 = min(x + 1, W - 1);
    const int y1 = min(y + 1, H - 1);
    const size_t r0 = (size_t)y * ld, r1 = (size_t)y1 * ld;
    const float a[4] = {__ldg(I0 + r0 + x), __ldg(I0 + r0 + x1), __ldg(I0 + r1 + x),
                        __ldg(I0 + r1 + x1)};
    const float b[4] = {__ldg(I1 + r0 + x), __ldg(I1 + r0 + x1), __ldg(I1 + r1 + x),
                        __ldg(I1 + r1 + x1)};
    const float wx[4] = {-0.25f, 0.25f, -0.25f, 0.25f};
    const float wy[4] = {-0.25f, -0.25f, 0.25f, 0.25f};
    float ax0 = 0.f, ax1 = 0.f, ay0 = 0.f, ay1 = 0.f, at0 = 0.f, at1 = 0.f;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        ax0 = __fadd_rn(ax0, __fmul_rn(wx[d], a[d]));
        ax1 = __fadd_rn(ax1, __fmul_rn(wx[d], b[d]));
        ay0 = __fadd_rn(ay0, __fmul_rn(wy[d], a[d]));
        ay1 = __fadd_rn(ay1, __fmul_rn(wy[d], b[d]));
        at0 = __fadd_rn(at0, __fmul_rn(0.25f, a[d]));
        at1 = __fadd_rn(at1, __fmul_rn(0.25f, b[d]));
    }
    Ix = __fadd_rn(ax0, ax1);
    Iy = __fadd_rn(ay0, ay1);
    It = __fsub_rn(at1, at0);
}
#endif

}  // namespace hs
