// hs_cg.cu -- Horn-Schunck as a linear system: the operator powers behind an s-step
// Krylov solver (HSMatrixPowers) and the 2x2 block-Jacobi preconditioner
// (ApplyHSPreconditioner).
//
// Matrix powers: V[0] = r, V[s] = M V[s-1] with
//   M (u, v) = (Ix g, Iy g) + lam * (deg*mid - sum of the present 4-neighbours), g = Ix u + Iy v
// evaluated in the operation order of HSMatrixPowers.cpp:72-106 (one rounding each), so the
// result is bit-identical to the reference's FP32 semantics.  Every power is an output, so
// a pass cannot skip writes; what temporal blocking saves is the reads: a CTA loads a
// (64 + 8) x (32 + 2T) tile of u, v, Ix, Iy once into shared memory, advances it T powers
// there (the valid region shrinks by one cell per power) and writes each power's 64 x 32 core.
// Per power that is 8 B/px written plus (16 B/px x halo overhead) / T read, against
// 24 B/px for one launch per power.
#include <algorithm>

#include "hs_common.cuh"

namespace hs {

constexpr int kMpTX = 64;       // output tile width
constexpr int kMpTY = 32;       // output tile height
constexpr int kMpHX = 4;        // halo columns each side (>= depth; 16-byte aligned loads)
constexpr int kMpMaxDepth = 4;  // powers per pass
constexpr int kMpThreads = 256;

template <int D>
struct MpGeo {
    static constexpr int EX = kMpTX + 2 * kMpHX;  // tile width with halo
    static constexpr int EY = kMpTY + 2 * D;      // tile height with halo
    static constexpr int N = EX * EY;
    static constexpr int smem_bytes = 6 * N * (int)sizeof(float);  // Ix, Iy, u0, v0, u1, v1
};

// One power at one cell from the previous power in shared memory (row stride E); the
// neighbour tests use image coordinates, as the template's element_id tests do.
__device__ __forceinline__ void mp_cell(const float *u, const float *v, const float *Ix,
                                        const float *Iy, int c, int E, int x, int y, int H, int W,
                                        float lam, float &ur, float &vr) {
    const float um = u[c], vm = v[c], ix = Ix[c], iy = Iy[c];
    const float g = __fadd_rn(__fmul_rn(ix, um), __fmul_rn(iy, vm));
    ur = __fmul_rn(ix, g);
    vr = __fmul_rn(iy, g);
    const float nl = -lam;
    const float lu = __fmul_rn(lam, um), lv = __fmul_rn(lam, vm);
    if (x > 0) {
        ur = __fadd_rn(__fadd_rn(ur, __fmul_rn(nl, u[c - 1])), lu);
        vr = __fadd_rn(__fadd_rn(vr, __fmul_rn(nl, v[c - 1])), lv);
    }
    if (x < W - 1) {
        ur = __fadd_rn(__fadd_rn(ur, __fmul_rn(nl, u[c + 1])), lu);
        vr = __fadd_rn(__fadd_rn(vr, __fmul_rn(nl, v[c + 1])), lv);
    }
    if (y > 0) {
        ur = __fadd_rn(__fadd_rn(ur, __fmul_rn(nl, u[c - E])), lu);
        vr = __fadd_rn(__fadd_rn(vr, __fmul_rn(nl, v[c - E])), lv);
    }
    if (y < H - 1) {
        ur = __fadd_rn(__fadd_rn(ur, __fmul_rn(nl, u[c + E])), lu);
        vr = __fadd_rn(__fadd_rn(vr, __fmul_rn(nl, v[c + E])), lv);
    }
}

// One power over the tile region [x0, x0+SX) x [y0, y0+SY) (tile coordinates), flattened
// over the CTA's threads.  INTERIOR: the whole tile lies at least one cell inside the image,
// so every computed cell has its four neighbours and no test is needed.
template <int EX, int SX, int SY, bool INTERIOR>
__device__ __forceinline__ void mp_region(const float *u, const float *v, const float *sIx,
                                          const float *sIy, float *uo, float *vo, int x0, int y0,
                                          int tx0, int ty0, int H, int W, float lam) {
    for (int k = threadIdx.x; k < SX * SY; k += kMpThreads) {
        const int cy = y0 + k / SX, cx = x0 + k % SX;
        const int c = cy * EX + cx;
        float ur, vr;
        if constexpr (INTERIOR) {
            mp_cell(u, v, sIx, sIy, c, EX, 1, 1, 3, 3, lam, ur, vr);  // all neighbours present
        } else {
            const int x = tx0 + cx, y = ty0 + cy;
            if (x < 0 || x >= W || y < 0 || y >= H) continue;
            mp_cell(u, v, sIx, sIy, c, EX, x, y, H, W, lam, ur, vr);
        }
        uo[c] = ur;
        vo[c] = vr;
    }
}

// Power T of a pass of D (T = 1 .. D, unrolled at compile time): compute it over the
// region still needed by the later powers, then store its core.
template <int D, int T>
__device__ __forceinline__ void mp_power(float *sIx, float *sIy, float *su0, float *sv0, float *su1,
                                         float *sv1, bool interior, int tx0, int ty0, int H, int W,
                                         int ld, float lam, float *V0, float *V1, size_t pstride) {
    constexpr int EX = MpGeo<D>::EX;
    constexpr int M = D - T;  // power T is needed within M cells of the core
    constexpr int SX = kMpTX + 2 * M, SY = kMpTY + 2 * M;
    constexpr bool odd = T & 1;
    const float *u = odd ? su0 : su1, *v = odd ? sv0 : sv1;
    float *uo = odd ? su1 : su0, *vo = odd ? sv1 : sv0;
    if (interior)
        mp_region<EX, SX, SY, true>(u, v, sIx, sIy, uo, vo, kMpHX - M, D - M, tx0, ty0, H, W, lam);
    else
        mp_region<EX, SX, SY, false>(u, v, sIx, sIy, uo, vo, kMpHX - M, D - M, tx0, ty0, H, W, lam);
    __syncthreads();
    // store the core (the next power reads uo as well and writes the other buffer)
    float *out0 = V0 + (size_t)T * pstride, *out1 = V1 + (size_t)T * pstride;
    for (int k = threadIdx.x; k < (kMpTX / 4) * kMpTY; k += kMpThreads) {
        const int gx = k % (kMpTX / 4), cy = D + k / (kMpTX / 4);
        const int x = tx0 + kMpHX + 4 * gx, y = ty0 + cy;
        if (x >= W || y >= H) continue;
        const int c = cy * EX + kMpHX + 4 * gx;
        const size_t o = (size_t)y * ld + x;
        if (x + 4 <= W) {
            *reinterpret_cast<float4 *>(out0 + o) = *reinterpret_cast<const float4 *>(uo + c);
            *reinterpret_cast<float4 *>(out1 + o) = *reinterpret_cast<const float4 *>(vo + c);
        } else {
            for (int j = 0; j < W - x; ++j) {
                out0[o + j] = uo[c + j];
                out1[o + j] = vo[c + j];
            }
        }
    }
    if constexpr (T < D)
        mp_power<D, T + 1>(sIx, sIy, su0, sv0, su1, sv1, interior, tx0, ty0, H, W, ld, lam, V0, V1,
                           pstride);
}

// D powers: V[s0+1 .. s0+D] from V[s0].  Loads and stores move 16-byte groups (the tile's
// first column is a multiple of 4, rows start 16-byte aligned); tile cells outside the image
// load as 0 and are never read by an in-image cell (the neighbour tests skip them).
template <int D>
__global__ void __launch_bounds__(kMpThreads) mp_pass_kernel(float lam, const float *__restrict__ Ix,
                                                             const float *__restrict__ Iy,
                                                             const float *u_in, const float *v_in,
                                                             float *V0, float *V1, size_t pstride,
                                                             int H, int W, int ld) {
    using G = MpGeo<D>;
    constexpr int EX = G::EX, EY = G::EY, GX = EX / 4;
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    float *sIx = sm, *sIy = sm + G::N;
    float *su0 = sm + 2 * G::N, *sv0 = sm + 3 * G::N, *su1 = sm + 4 * G::N, *sv1 = sm + 5 * G::N;
    const int tx0 = blockIdx.x * kMpTX - kMpHX, ty0 = blockIdx.y * kMpTY - D;
    const bool interior = tx0 >= 1 && ty0 >= 1 && tx0 + EX <= W - 1 && ty0 + EY <= H - 1;
    for (int c = threadIdx.x; c < GX * EY; c += kMpThreads) {
        const int gx = c % GX, cy = c / GX;
        const int x = tx0 + 4 * gx, y = ty0 + cy;
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, p = a, q = a;
        if (x >= 0 && x + 4 <= ld && y >= 0 && y < H) {
            const size_t o = (size_t)y * ld + x;
            a = __ldg(reinterpret_cast<const float4 *>(Ix + o));
            b = __ldg(reinterpret_cast<const float4 *>(Iy + o));
            p = *reinterpret_cast<const float4 *>(u_in + o);
            q = *reinterpret_cast<const float4 *>(v_in + o);
        }
        const int k = cy * EX + 4 * gx;
        *reinterpret_cast<float4 *>(sIx + k) = a;
        *reinterpret_cast<float4 *>(sIy + k) = b;
        *reinterpret_cast<float4 *>(su0 + k) = p;
        *reinterpret_cast<float4 *>(sv0 + k) = q;
    }
    __syncthreads();
    mp_power<D, 1>(sIx, sIy, su0, sv0, su1, sv1, interior, tx0, ty0, H, W, ld, lam, V0, V1, pstride);
}

__device__ __forceinline__ void precond_px(float s2, float a, float d, float b, float e, float f,
                                           int x, int y, int H, int W, float &o0, float &o1) {
    // ApplyHSPreconditioner.cpp:49-68: one s per neighbour present
    if (x < W - 1) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    if (y < H - 1) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    if (x > 0) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    if (y > 0) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    const float det = __fsub_rn(__fmul_rn(a, d), __fmul_rn(b, b));
    if (fabsf(det) > 1e-15f) {
        o0 = __fdiv_rn(__fsub_rn(__fmul_rn(e, d), __fmul_rn(b, f)), det);
        o1 = __fdiv_rn(__fadd_rn(__fmul_rn(-b, e), __fmul_rn(a, f)), det);
    } else {
        o0 = e;
        o1 = f;
    }
}

// Four pixels per thread with 16-byte accesses (rows start 16-byte aligned, ld % 4 == 0);
// the last group of a row may hold columns past W, which are neither read nor written.
__global__ void __launch_bounds__(256) precond_kernel(float s2, const float *__restrict__ diag0,
                                                      const float *__restrict__ diag1,
                                                      const float *__restrict__ offdiag,
                                                      const float *__restrict__ x0,
                                                      const float *__restrict__ x1, int H, int W,
                                                      int ld, float *__restrict__ y0,
                                                      float *__restrict__ y1) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = 4 * gx;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * ld + x;
    if (x + 4 <= W) {
        const float4 A = __ldg(reinterpret_cast<const float4 *>(diag0 + i));
        const float4 Dd = __ldg(reinterpret_cast<const float4 *>(diag1 + i));
        const float4 B = __ldg(reinterpret_cast<const float4 *>(offdiag + i));
        const float4 E = __ldg(reinterpret_cast<const float4 *>(x0 + i));
        const float4 F = __ldg(reinterpret_cast<const float4 *>(x1 + i));
        float4 o0, o1;
        precond_px(s2, A.x, Dd.x, B.x, E.x, F.x, x, y, H, W, o0.x, o1.x);
        precond_px(s2, A.y, Dd.y, B.y, E.y, F.y, x + 1, y, H, W, o0.y, o1.y);
        precond_px(s2, A.z, Dd.z, B.z, E.z, F.z, x + 2, y, H, W, o0.z, o1.z);
        precond_px(s2, A.w, Dd.w, B.w, E.w, F.w, x + 3, y, H, W, o0.w, o1.w);
        *reinterpret_cast<float4 *>(y0 + i) = o0;
        *reinterpret_cast<float4 *>(y1 + i) = o1;
    } else {
        for (int j = 0; j < W - x; ++j) {
            float o0, o1;
            precond_px(s2, __ldg(diag0 + i + j), __ldg(diag1 + i + j), __ldg(offdiag + i + j),
                       __ldg(x0 + i + j), __ldg(x1 + i + j), x + j, y, H, W, o0, o1);
            y0[i + j] = o0;
            y1[i + j] = o1;
        }
    }
}

template <int D>
static hs_status launch_mp(float lam, const float *Ix, const float *Iy, const float *u,
                           const float *v, float *V0, float *V1, size_t pstride, int H, int W,
                           int ld, cudaStream_t s) {
    static bool attr[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(mp_pass_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           MpGeo<D>::smem_bytes));
        attr[dev] = true;
    }
    const dim3 grid((unsigned)((W + kMpTX - 1) / kMpTX), (unsigned)((H + kMpTY - 1) / kMpTY));
    mp_pass_kernel<D><<<grid, kMpThreads, MpGeo<D>::smem_bytes, s>>>(lam, Ix, Iy, u, v, V0, V1,
                                                                      pstride, H, W, ld);
    HS_LAUNCH_CHECK("mp_pass_kernel");
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" {

hs_status hs_matrix_powers(float lam, const float *Ix, const float *Iy, const float *r0,
                           const float *r1, int H, int W, int ld, int steps, float *V0, float *V1,
                           size_t power_stride, const hs_config *cfg, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *pl[6] = {Ix, Iy, r0, r1, V0, V1};
    const char *nm[6] = {"Ix", "Iy", "r0", "r1", "V0", "V1"};
    for (int k = 0; k < 6; ++k)
        if ((st = check_plane(pl[k], nm[k])) != HS_OK) return st;
    if (steps < 1) HS_FAIL(HS_ERR_INVALID_ARG, "steps=%d must be >= 1", steps);
    if (power_stride < (size_t)H * ld || power_stride % 4 != 0)
        HS_FAIL(HS_ERR_INVALID_ARG, "power_stride=%zu must be >= H*ld and a multiple of 4", power_stride);
    int depth = (cfg && cfg->sweeps_per_pass > 0) ? cfg->sweeps_per_pass : kMpMaxDepth;
    if (depth > kMpMaxDepth) HS_FAIL(HS_ERR_INVALID_ARG, "sweeps_per_pass=%d outside 1..%d", depth, kMpMaxDepth);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t row = (size_t)W * sizeof(float), pitch = (size_t)ld * sizeof(float);
    if (V0 != r0) HS_CUDA_CHECK(cudaMemcpy2DAsync(V0, pitch, r0, pitch, row, H, cudaMemcpyDeviceToDevice, s));
    if (V1 != r1) HS_CUDA_CHECK(cudaMemcpy2DAsync(V1, pitch, r1, pitch, row, H, cudaMemcpyDeviceToDevice, s));
    for (int s0 = 0; s0 + 1 < steps; s0 += depth) {
        const int d = std::min(depth, steps - 1 - s0);
        float *b0 = V0 + (size_t)s0 * power_stride, *b1 = V1 + (size_t)s0 * power_stride;
        switch (d) {  // this pass's depth
            case 1: st = launch_mp<1>(lam, Ix, Iy, b0, b1, b0, b1, power_stride, H, W, ld, s); break;
            case 2: st = launch_mp<2>(lam, Ix, Iy, b0, b1, b0, b1, power_stride, H, W, ld, s); break;
            case 3: st = launch_mp<3>(lam, Ix, Iy, b0, b1, b0, b1, power_stride, H, W, ld, s); break;
            default: st = launch_mp<4>(lam, Ix, Iy, b0, b1, b0, b1, power_stride, H, W, ld, s); break;
        }
        if (st != HS_OK) return st;
    }
    return HS_OK;
}

hs_status hs_apply_hs_preconditioner(float s2, const float *diag0, const float *diag1,
                                     const float *offdiag, const float *x0, const float *x1,
                                     int H, int W, int ld, float *y0, float *y1, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *pl[7] = {diag0, diag1, offdiag, x0, x1, y0, y1};
    const char *nm[7] = {"diag0", "diag1", "offdiag", "x0", "x1", "y0", "y1"};
    for (int k = 0; k < 7; ++k)
        if ((st = check_plane(pl[k], nm[k])) != HS_OK) return st;
    const int groups = (W + 3) / 4;
    const dim3 grid((unsigned)((groups + 63) / 64), (unsigned)((H + 3) / 4));
    precond_kernel<<<grid, dim3(64, 4), 0, (cudaStream_t)stream>>>(s2, diag0, diag1, offdiag, x0, x1,
                                                                    H, W, ld, y0, y1);
    HS_LAUNCH_CHECK("precond_kernel");
    return HS_OK;
}

}  // extern "C"
