// hs_cg.cu -- Horn-Schunck as a linear system: the operator powers behind an s-step
// Krylov solver (HSMatrixPowers) and the 2x2 block-Jacobi preconditioner
// (ApplyHSPreconditioner).
//
// Matrix powers: V[0] = r, V[s] = M V[s-1] with
//   M (u, v) = (Ix g, Iy g) + lam * (deg*mid - sum of the present 4-neighbours), g = Ix u + Iy v
// evaluated in the operation order of HSMatrixPowers.cpp:72-106 (one rounding each), so the
// result is bit-identical to the reference's FP32 semantics.  Every power is an output, so
// a pass cannot skip writes; what temporal blocking saves is the reads.  A pass of D powers
// streams the strip down the image like the Jacobi sweep (hs_stream4.cuh): a warp owns a
// 128-column strip (4 columns per lane) of a segment of rows, D stages form a register
// pipeline (stage s turns row n of power s0+s into row n-1 of power s0+s+1 and writes it),
// each stage keeps its two previous input rows in registers, and only the two lane-edge
// columns cross lanes (shuffles).  Per power that is 8 B/px written plus 16 B/px / D read
// (plus the strips' 4-column halos).
#include <algorithm>

#include "hs_stream.cuh"

namespace hs {

constexpr int kMpMaxDepth = 4;                     // powers per pass
constexpr int kMpCols = 128;                       // strip width (4 columns per lane)
constexpr int kMpHalo = 4;                         // >= depth; keeps chunks 16-byte aligned
constexpr int kMpStrip = kMpCols - 2 * kMpHalo;    // output columns per strip
constexpr int kMpPrefetch = 2;                     // rows in flight per warp
constexpr int kMpPlanes = 4;                       // u, v, Ix, Iy
constexpr int kMpWarps = 1;                        // warps per CTA (each warp is a work item)
constexpr int kMpResWarps = 12;                    // resident warps per SM the registers allow

template <int D>
struct MpGeo {
    // ring of rows: stage s at step k reads Ix, Iy of row k-s-1, so rows k-D .. k+prefetch
    static constexpr int slots = D + 1 + kMpPrefetch;
    static constexpr int warp_floats = slots * kMpPlanes * kMpCols;
    static constexpr int smem_bytes = kMpWarps * warp_floats * (int)sizeof(float);
};

struct MpParams {
    const float *Ix, *Iy, *u_in, *v_in;
    float *V0, *V1;     // power s0 of the pass (V[s0]); power s0+j at + j * pstride
    size_t pstride;
    int H, W, ld, seg_rows, nstrips, nitems;
    float lam;
    int copy0;          // also write the input rows as power s0 (V[0] = r on the first pass)
};

// One cell of one power (HSMatrixPowers.cpp:72-106 order): m = (u, v) at the cell,
// l / r / up / dn its neighbours, present per the flags.  The u and v chains run as one
// packed pair: the products are scalar (mul2r: rounded on their own, never fused) and the
// adds packed (add.rn.f32x2: each half one IEEE add), so every operation rounds exactly as
// the template's scalar code.
__device__ __forceinline__ float2 mp_cell(float ix, float iy, float2 m, float2 l, float2 r,
                                          float2 up, float2 dn, bool hl, bool hr, bool hu, bool hd,
                                          float lam) {
    const float g = __fadd_rn(__fmul_rn(ix, m.x), __fmul_rn(iy, m.y));
    float2 o = mul2r(f2(ix, iy), f2(g, g));
    const float2 nl = f2(-lam, -lam);
    const float2 lm = mul2r(f2(lam, lam), m);
    if (hl) o = add2(add2(o, mul2r(nl, l)), lm);
    if (hr) o = add2(add2(o, mul2r(nl, r)), lm);
    if (hu) o = add2(add2(o, mul2r(nl, up)), lm);
    if (hd) o = add2(add2(o, mul2r(nl, dn)), lm);
    return o;
}

// A stage's window: its two previous input rows (4 columns of u and v), the middle row's
// neighbours across the lane edges.
struct MpWin {
    float4 uu, vu;        // row n-2
    float4 um, vm;        // row n-1
    float ml_u, ml_v;     // row n-1, column xa-1
    float mr_u, mr_v;     // row n-1, column xa+4
};

__device__ __forceinline__ float4 f4get(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float f4at(const float4 &a, int j) {
    return j == 0 ? a.x : (j == 1 ? a.y : (j == 2 ? a.z : a.w));
}

// 12 warps per SM: the depth-4 pass needs up to 168 registers and 14 KB of shared memory per
// warp.  One-warp CTAs free a slot as soon as its item ends; under programmatic dependent
// launch the next pass's items take it while the rest of this pass finishes.
template <int D>
__global__ void __launch_bounds__(kMpWarps * 32, kMpResWarps / kMpWarps) mp_stream_kernel(const MpParams p) {
    using G = MpGeo<D>;
    extern __shared__ float4 sm4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *ring = reinterpret_cast<float *>(sm4) + warp * G::warp_floats;
    griddep_launch_dependents();
    griddep_wait();  // the previous pass (its powers are this pass's input) has completed
    const int item = blockIdx.x * kMpWarps + warp;
    if (item >= p.nitems) return;  // warp-uniform
    const int strip = item % p.nstrips, seg = item / p.nstrips;
    const int xa = strip * kMpStrip - kMpHalo + 4 * lane;  // first of the lane's 4 columns
    const int lcol = (xa >= 0 && xa + 4 <= p.ld) ? xa : 0;  // any in-bounds chunk otherwise
    const int vlo = strip * kMpStrip, vhi = min(vlo + kMpStrip, p.W);
    unsigned st = 0u;  // bit j: column xa+j is stored by this strip
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (xa + j >= vlo && xa + j < vhi) st |= 1u << j;
    const int y_start = seg * p.seg_rows, y_end = min(p.H, y_start + p.seg_rows);
    const int k0 = max(0, y_start - D), k_end = y_end - 1 + D;
    const int last_row = y_end - 1 + D;  // rows past it are never needed

    auto issue = [&](int row) {
        const int slot = ((row % G::slots) + G::slots) % G::slots;
        const int r = min(max(row, 0), p.H - 1);
        const size_t off = (size_t)r * p.ld + lcol;
        float *b = ring + slot * (kMpPlanes * kMpCols) + 4 * lane;
        cp_async16(b + 0 * kMpCols, p.u_in + off);
        cp_async16(b + 1 * kMpCols, p.v_in + off);
        cp_async16(b + 2 * kMpCols, p.Ix + off);
        cp_async16(b + 3 * kMpCols, p.Iy + off);
        cp_async_commit();
    };
    auto store = [&](float *U, float *V, int r, float4 a, float4 b) {
        if (r < y_start || r >= y_end || st == 0u) return;
        const size_t o = (size_t)r * p.ld + xa;
        if (st == 15u) {
            *reinterpret_cast<float4 *>(U + o) = a;
            *reinterpret_cast<float4 *>(V + o) = b;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (st & (1u << j)) {
                    U[o + j] = f4at(a, j);
                    V[o + j] = f4at(b, j);
                }
        }
    };

    MpWin w[D];
#pragma unroll
    for (int s = 0; s < D; ++s) w[s] = MpWin{};
#pragma unroll
    for (int i = 0; i < kMpPrefetch; ++i) issue(k0 + i);
    for (int k = k0; k <= k_end; ++k) {
        issue(min(k + kMpPrefetch, last_row));
        cp_async_wait<kMpPrefetch>();
        const float *row_k = ring + (k % G::slots) * (kMpPlanes * kMpCols) + 4 * lane;
        float4 cu = f4get(row_k), cv = f4get(row_k + kMpCols);  // row k of power s0
        if (p.copy0) store(p.V0, p.V1, k, cu, cv);
#pragma unroll
        for (int s = 0; s < D; ++s) {
            MpWin &q = w[s];
            const int n = k - s;     // arriving row of power s0+s
            const int r = n - 1;     // the row this stage emits (power s0+s+1)
            const float *row_r = ring + (((r % G::slots) + G::slots) % G::slots) * (kMpPlanes * kMpCols) + 4 * lane;
            const float4 ix = f4get(row_r + 2 * kMpCols), iy = f4get(row_r + 3 * kMpCols);
            const bool hu = r > 0, hd = r < p.H - 1;
            float4 ou, ov;
            float *o_u = &ou.x, *o_v = &ov.x;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = xa + j;
                const float2 l = j == 0 ? f2(q.ml_u, q.ml_v) : f2(f4at(q.um, j - 1), f4at(q.vm, j - 1));
                const float2 rr = j == 3 ? f2(q.mr_u, q.mr_v) : f2(f4at(q.um, j + 1), f4at(q.vm, j + 1));
                const float2 o = mp_cell(f4at(ix, j), f4at(iy, j), f2(f4at(q.um, j), f4at(q.vm, j)), l, rr,
                                         f2(f4at(q.uu, j), f4at(q.vu, j)), f2(f4at(cu, j), f4at(cv, j)),
                                         x > 0, x < p.W - 1, hu, hd, p.lam);
                o_u[j] = o.x;
                o_v[j] = o.y;
            }
            // advance the window: row n becomes the middle row, with its lane-edge neighbours
            q.uu = q.um;
            q.vu = q.vm;
            q.um = cu;
            q.vm = cv;
            q.ml_u = __shfl_up_sync(kFull, cu.w, 1);
            q.ml_v = __shfl_up_sync(kFull, cv.w, 1);
            q.mr_u = __shfl_down_sync(kFull, cu.x, 1);
            q.mr_v = __shfl_down_sync(kFull, cv.x, 1);
            store(p.V0 + (size_t)(s + 1) * p.pstride, p.V1 + (size_t)(s + 1) * p.pstride, r, ou, ov);
            cu = ou;
            cv = ov;
        }
    }
    cp_async_wait<0>();
}

template <int D>
static hs_status launch_mp(const MpParams &pp, cudaStream_t s) {
    static bool attr[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(mp_stream_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           MpGeo<D>::smem_bytes));
        attr[dev] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((pp.nitems + kMpWarps - 1) / kMpWarps));
    cfg.blockDim = dim3(kMpWarps * 32);
    cfg.dynamicSmemBytes = MpGeo<D>::smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute a[1];
    a[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    a[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = a;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, mp_stream_kernel<D>, pp));
    return HS_OK;
}

__device__ __forceinline__ void precond_px(float s2, float a, float d, float b, float e, float f,
                                           int x, int y, int H, int W, float &o0, float &o1) {
    // ApplyHSPreconditioner.cpp:49-68: one s per neighbour present
    if (x < W - 1) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    if (y < H - 1) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    if (x > 0) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    if (y > 0) { a = __fadd_rn(a, s2); d = __fadd_rn(d, s2); }
    const float det = __fsub_rn(__fmul_rn(a, d), __fmul_rn(b, b));
    // the template's fabs(det) > 1e-15 compares in double: float(1e-15) lies above 1e-15
    if ((double)fabsf(det) > 1e-15) {
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
    // segments: about one wave of resident warps over all strips, at least 8 rows
    const int nstrips = (W + kMpStrip - 1) / kMpStrip;
    const long target = (long)sm_count() * kMpResWarps;
    const long nseg = std::max(1L, (target + nstrips - 1) / nstrips);
    const int seg_rows = (cfg && cfg->rows_per_segment > 0)
                             ? std::min(H, cfg->rows_per_segment)
                             : std::min(H, std::max(8, (int)((H + nseg - 1) / nseg)));
    const int nitems = nstrips * ((H + seg_rows - 1) / seg_rows);
    if (steps == 1) {  // V[0] = r only
        if (V0 != r0) HS_CUDA_CHECK(cudaMemcpy2DAsync(V0, pitch, r0, pitch, row, H, cudaMemcpyDeviceToDevice, s));
        if (V1 != r1) HS_CUDA_CHECK(cudaMemcpy2DAsync(V1, pitch, r1, pitch, row, H, cudaMemcpyDeviceToDevice, s));
        return HS_OK;
    }
    for (int s0 = 0; s0 + 1 < steps; s0 += depth) {
        const int d = std::min(depth, steps - 1 - s0);
        MpParams pp;
        pp.Ix = Ix;
        pp.Iy = Iy;
        pp.V0 = V0 + (size_t)s0 * power_stride;
        pp.V1 = V1 + (size_t)s0 * power_stride;
        // the first pass reads r itself and writes it out as V[0] (unless r is V[0])
        pp.u_in = s0 == 0 ? r0 : pp.V0;
        pp.v_in = s0 == 0 ? r1 : pp.V1;
        pp.copy0 = (s0 == 0 && (V0 != r0 || V1 != r1)) ? 1 : 0;
        pp.pstride = power_stride;
        pp.H = H;
        pp.W = W;
        pp.ld = ld;
        pp.seg_rows = seg_rows;
        pp.nstrips = nstrips;
        pp.nitems = nitems;
        pp.lam = lam;
        switch (d) {  // this pass's depth
            case 1: st = launch_mp<1>(pp, s); break;
            case 2: st = launch_mp<2>(pp, s); break;
            case 3: st = launch_mp<3>(pp, s); break;
            default: st = launch_mp<4>(pp, s); break;
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
