// hs_ops.cu -- library plumbing and the structured-grid operator kernels of libhsflow:
// the generic clamp-to-edge stencil (Stencil2DMVM), the pointwise Array2D operators and
// the fused Horn-Schunck derivative pass.
//
// All kernels here are HBM-bound one-pass maps over FP32 planes.  They use one rounding
// per operation (__fmul_rn / __fadd_rn / __fdiv_rn, which the compiler never contracts),
// in the reference program's order, so their results equal the reference's FP32
// semantics bit for bit.
#include <cstring>
#include <mutex>
#include <vector>

#include "hs_common.cuh"

namespace hs {

static thread_local char g_last_error[512];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

void clear_error() { g_last_error[0] = '\0'; }

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

// ------------------------------------------------------------------ kernels

struct StencilTaps {
    float w[HS_MAX_TAPS];
    int ox[HS_MAX_TAPS];
    int oy[HS_MAX_TAPS];
    int n;
};

// Stencil2DMVM.cpp:37-48: y = 0; for each tap: clamp both coordinates, y += S[d] * x.
__global__ void __launch_bounds__(256) stencil2d_kernel(const __grid_constant__ StencilTaps taps,
                                                        const float *__restrict__ in,
                                                        float *__restrict__ out, int H, int W,
                                                        int ld) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float acc = 0.0f;
    for (int d = 0; d < taps.n; ++d) {
        const int xx = min(max(x + taps.ox[d], 0), W - 1);
        const int yy = min(max(y + taps.oy[d], 0), H - 1);
        acc = __fadd_rn(acc, __fmul_rn(taps.w[d], __ldg(in + (size_t)yy * ld + xx)));
    }
    out[(size_t)y * ld + x] = acc;
}

__device__ __forceinline__ float apply_op(int op, float b, float c) {
    switch (op) {
        case HS_OP_ADD: return __fadd_rn(b, c);
        case HS_OP_SUB: return __fsub_rn(b, c);
        case HS_OP_MUL: return __fmul_rn(b, c);
        default: return __fdiv_rn(b, c);
    }
}

// mode 0: a = b op c; mode 1: a = b op s; mode 2: a = s op b; mode 3: a = b.
__global__ void __launch_bounds__(256) pointwise_kernel(int mode, int op,
                                                        const float *__restrict__ b,
                                                        const float *__restrict__ c, float s,
                                                        float *__restrict__ a, int H, int W,
                                                        int ld) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * ld + x;
    float r;
    if (mode == 0) r = apply_op(op, b[i], c[i]);
    else if (mode == 1) r = apply_op(op, b[i], s);
    else if (mode == 2) r = apply_op(op, s, b[i]);
    else r = b[i];
    a[i] = r;
}

// Horn-Schunck 2x2x2 derivatives, one pass (hs_derivs_at in hs_common.cuh).
__global__ void __launch_bounds__(256) derivs_kernel(const float *__restrict__ I0,
                                                     const float *__restrict__ I1,
                                                     float *__restrict__ Ix,
                                                     float *__restrict__ Iy,
                                                     float *__restrict__ It, int H, int W,
                                                     int ld) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * ld + x;
    hs_derivs_at(I0, I1, x, y, H, W, ld, Ix[i], Iy[i], It[i]);
}

static inline dim3 grid2d(int H, int W, dim3 block) {
    return dim3((unsigned)((W + block.x - 1) / block.x), (unsigned)((H + block.y - 1) / block.y));
}

static hs_status launch_pointwise(int mode, int op, const float *b, const float *c, float s,
                                  float *a, int H, int W, int ld, void *stream) {
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    if ((st = check_plane(b, "b")) != HS_OK) return st;
    if (mode == 0 && (st = check_plane(c, "c")) != HS_OK) return st;
    if ((st = check_plane(a, "a")) != HS_OK) return st;
    if (mode != 3 && (op < HS_OP_ADD || op > HS_OP_DIV))
        HS_FAIL(HS_ERR_INVALID_ARG, "op=%d is not one of HS_OP_ADD..HS_OP_DIV", op);
    dim3 block(64, 4);
    pointwise_kernel<<<grid2d(H, W, block), block, 0, (cudaStream_t)stream>>>(mode, op, b, c, s, a,
                                                                              H, W, ld);
    HS_LAUNCH_CHECK("pointwise_kernel");
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" {

const char *hs_status_string(hs_status status) {
    switch (status) {
        case HS_OK: return "HS_OK";
        case HS_ERR_INVALID_ARG: return "HS_ERR_INVALID_ARG: invalid argument";
        case HS_ERR_ALIGNMENT: return "HS_ERR_ALIGNMENT: plane pointer or leading dimension misaligned";
        case HS_ERR_WORKSPACE: return "HS_ERR_WORKSPACE: workspace missing or too small";
        case HS_ERR_CUDA: return "HS_ERR_CUDA: CUDA runtime error";
        case HS_ERR_TIMEOUT: return "HS_ERR_TIMEOUT: bounded device wait expired";
        case HS_ERR_UNSUPPORTED: return "HS_ERR_UNSUPPORTED: not supported by this build";
        case HS_ERR_NO_DEVICE: return "HS_ERR_NO_DEVICE: no usable sm_100 device";
    }
    return "unknown hs_status";
}

const char *hs_last_error(void) { return g_last_error; }

int hs_version(void) { return 100; }

hs_status hs_stencil2d(const float *weights, const int *offx, const int *offy, int ntaps,
                       const float *in, float *out, int H, int W, int ld, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    if (!weights || !offx || !offy) HS_FAIL(HS_ERR_INVALID_ARG, "stencil taps are NULL");
    if (ntaps < 1 || ntaps > HS_MAX_TAPS)
        HS_FAIL(HS_ERR_INVALID_ARG, "ntaps=%d outside 1..%d", ntaps, HS_MAX_TAPS);
    if ((st = check_plane(in, "in")) != HS_OK) return st;
    if ((st = check_plane(out, "out")) != HS_OK) return st;
    if (in == out) HS_FAIL(HS_ERR_INVALID_ARG, "in and out must differ");
    StencilTaps taps;
    memset(&taps, 0, sizeof(taps));
    for (int d = 0; d < ntaps; ++d) {
        taps.w[d] = weights[d];
        taps.ox[d] = offx[d];
        taps.oy[d] = offy[d];
    }
    taps.n = ntaps;
    dim3 block(64, 4);
    stencil2d_kernel<<<grid2d(H, W, block), block, 0, (cudaStream_t)stream>>>(taps, in, out, H, W,
                                                                              ld);
    HS_LAUNCH_CHECK("stencil2d_kernel");
    return HS_OK;
}

hs_status hs_array2d_op(int op, const float *b, const float *c, float *a, int H, int W, int ld,
                        void *stream) {
    clear_error();
    return launch_pointwise(0, op, b, c, 0.f, a, H, W, ld, stream);
}

hs_status hs_array2d_scalar_op(int op, const float *b, float s, float *a, int H, int W, int ld,
                               void *stream) {
    clear_error();
    return launch_pointwise(1, op, b, nullptr, s, a, H, W, ld, stream);
}

hs_status hs_scalar_array2d_op(int op, float s, const float *b, float *a, int H, int W, int ld,
                               void *stream) {
    clear_error();
    return launch_pointwise(2, op, b, nullptr, s, a, H, W, ld, stream);
}

hs_status hs_array2d_copy(const float *b, float *a, int H, int W, int ld, void *stream) {
    clear_error();
    return launch_pointwise(3, 0, b, nullptr, 0.f, a, H, W, ld, stream);
}

hs_status hs_derivs(const float *I0, const float *I1, int H, int W, int ld, float *Ix, float *Iy,
                    float *It, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *planes[5] = {I0, I1, Ix, Iy, It};
    const char *names[5] = {"I0", "I1", "Ix", "Iy", "It"};
    for (int i = 0; i < 5; ++i)
        if ((st = check_plane(planes[i], names[i])) != HS_OK) return st;
    dim3 block(64, 4);
    derivs_kernel<<<grid2d(H, W, block), block, 0, (cudaStream_t)stream>>>(I0, I1, Ix, Iy, It, H,
                                                                          W, ld);
    HS_LAUNCH_CHECK("derivs_kernel");
    return HS_OK;
}

}  // extern "C"
