// hs_sweep.cu -- the temporally blocked Horn-Schunck Jacobi sweep.
//
// One pass over HBM runs T sweeps.  Each warp owns a work item: a 64-column strip
// (2 adjacent columns per lane, loaded as float2) of a segment of rows.  The warp
// streams the segment's rows downward; row k enters stage 0 at step k, and stage s
// (1..T) emits sweep s of row k-s at the same step, so the T sweeps form a register
// pipeline down the strip:
//   - horizontal neighbours come from warp shuffles (only the lane-edge column moves),
//   - vertical neighbours come from a three-row rolling window kept in registers as
//     partial sums (exact mode: tap-ordered partial accumulators),
//   - the coefficient rows (Ix, Iy, It and the per-pixel denominator or its reciprocal)
//     sit in a per-warp shared-memory ring, filled by cp.async several rows ahead, so
//     global loads overlap the arithmetic of earlier rows.
// A strip loads `halo` extra columns each side and outputs the middle 64 - 2*halo; a
// segment starts T rows early; both are the temporal-blocking halo.  Warps never
// synchronise with each other: each lane reads only the shared-memory words it wrote.
//
// Clamp-to-edge boundaries (Stencil2DMVM.cpp:40-47): a neighbour outside the image is
// the pixel itself.  Horizontally the lane substitutes its own value; at the top the
// window of row 0 is seeded from row 0; at the bottom the missing row below H-1 is
// replaced by row H-1 held in the window.
//
// Exact mode (fast_math = 0) reproduces the reference program's FP32 operations one
// rounding at a time in its order: ubar = sum over the 8 taps in row-major order from
// 0; t = ((Ix*ubar + Iy*vbar) + It) / ((alpha2 + Ix*Ix) + Iy*Iy); u = ubar - Ix*t.
// Fast mode factors the average into edge and corner sums, uses fused multiply-adds
// and multiplies by a reciprocal of the denominator computed once per row per pass.
#include <algorithm>

#include "hs_common.cuh"

namespace hs {

constexpr int kWarpCols = 64;      // columns per strip (2 per lane)
constexpr int kPrefetch = 3;       // rows in flight per warp
constexpr int kWarpsPerBlock = 4;  // independent warps per CTA
constexpr int kPlanes = 6;         // ring planes: u, v, Ix, Iy, It, aux
constexpr unsigned kFull = 0xffffffffu;

template <int T>
struct Geo {
    static constexpr int halo = (T + 1) & ~1;                 // even, so lanes load float2
    static constexpr int strip = kWarpCols - 2 * halo;        // output columns per strip
    static constexpr int slots = T + 1 + kPrefetch;           // ring rows per warp
    static constexpr int ring_floats = slots * kPlanes * kWarpCols;
    static constexpr int smem_bytes = kWarpsPerBlock * ring_floats * (int)sizeof(float);
};

struct SweepParams {
    const float *Ix, *Iy, *It;
    const float *u_in, *v_in;
    float *u_out, *v_out;
    int H, W, ld;
    float alpha2;
    float we, wc;  // edge and corner weights of the average
    int seg_rows;
    int nstrips;
    int nitems;
};

__device__ __forceinline__ void cp_async8(float *smem, const float *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// Programmatic dependent launch: let the next pass's CTAs be scheduled early; wait for
// the previous pass (all of its memory operations) before touching any input.
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Issue the async copy of input row `row` (clamped into the image) into ring slot `slot`.
__device__ __forceinline__ void issue_row(float *ring, int slot, int row, const SweepParams &p,
                                          int lc, int lane) {
    row = min(max(row, 0), p.H - 1);
    const size_t off = (size_t)row * p.ld + lc;
    float *base = ring + slot * (kPlanes * kWarpCols) + 2 * lane;
    cp_async8(base + 0 * kWarpCols, p.u_in + off);
    cp_async8(base + 1 * kWarpCols, p.v_in + off);
    cp_async8(base + 2 * kWarpCols, p.Ix + off);
    cp_async8(base + 3 * kWarpCols, p.Iy + off);
    cp_async8(base + 4 * kWarpCols, p.It + off);
    cp_async_commit();
}

__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }

template <int T, bool FAST>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (T <= 4 ? 4 : 2))
    hs_stream_kernel(const SweepParams p) {
    using G = Geo<T>;
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *ring = reinterpret_cast<float *>(smem4) + warp * G::ring_floats;

    griddep_launch_dependents();
    griddep_wait();

    const int item = blockIdx.x * kWarpsPerBlock + warp;
    if (item >= p.nitems) return;  // warp-uniform
    const int strip = item % p.nstrips;
    const int seg = item / p.nstrips;
    const int x0 = strip * G::strip - G::halo;
    const int xa = x0 + 2 * lane, xb = xa + 1;
    // Column pair each lane loads: its own when it starts inside the image (xa is even
    // and ld is a multiple of 4, so xa + 1 < ld), any in-bounds pair otherwise -- columns
    // outside the image never feed a stored pixel.
    const int lc = (xa >= 0 && xa < p.W) ? xa : 0;
    const bool a_first = (xa == 0), a_last = (xa == p.W - 1), b_last = (xb == p.W - 1);
    const int vlo = strip * G::strip, vhi = min(vlo + G::strip, p.W);
    const bool st_a = (xa >= vlo && xa < vhi), st_b = (xb >= vlo && xb < vhi);
    const int y_start = seg * p.seg_rows;
    const int y_end = min(p.H, y_start + p.seg_rows);
    const int k0 = max(0, y_start - T);
    const int k_end = y_end - 1 + T;
    const float we = p.we, wc = p.wc;

    // Per-stage window state, [stage][plane u/v][column a/b].
    // fast:  cm = centre of the mid row, hm = its horizontal pair sum,
    //        E = c(up) + h(mid) (edge partial), C = h(up) (corner partial).
    // exact: A0 = accumulator of the next row holding its up taps, A1 = accumulator of
    //        the mid row holding its up and mid taps, lm/cm/rm = the mid row's values.
    float s0[T][2][2], s1[T][2][2], s2[T][2][2], s3[T][2][2], s4[T][2][2];
#pragma unroll
    for (int s = 0; s < T; ++s)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int j = 0; j < 2; ++j) s0[s][q][j] = s1[s][q][j] = s2[s][q][j] = s3[s][q][j] = s4[s][q][j] = 0.f;

#pragma unroll
    for (int i = 0; i < kPrefetch; ++i) issue_row(ring, i, k0 + i, p, lc, lane);

    int kslot = 0;
    for (int k = k0; k <= k_end; ++k) {
        int pslot = kslot + kPrefetch;
        if (pslot >= G::slots) pslot -= G::slots;
        issue_row(ring, pslot, k + kPrefetch, p, lc, lane);
        cp_async_wait<kPrefetch>();

        // ---- stage 0: row k arrives; derive the per-pixel denominator term.
        float *sl = ring + kslot * (kPlanes * kWarpCols) + 2 * lane;
        const float2 u2 = lds2(sl), v2 = lds2(sl + kWarpCols);
        {
            const float2 ix = lds2(sl + 2 * kWarpCols), iy = lds2(sl + 3 * kWarpCols);
            float2 aux;
            if constexpr (FAST) {
                aux.x = 1.0f / fmaf(iy.x, iy.x, fmaf(ix.x, ix.x, p.alpha2));
                aux.y = 1.0f / fmaf(iy.y, iy.y, fmaf(ix.y, ix.y, p.alpha2));
            } else {
                aux.x = __fadd_rn(__fadd_rn(p.alpha2, __fmul_rn(ix.x, ix.x)), __fmul_rn(iy.x, iy.x));
                aux.y = __fadd_rn(__fadd_rn(p.alpha2, __fmul_rn(ix.y, ix.y)), __fmul_rn(iy.y, iy.y));
            }
            *reinterpret_cast<float2 *>(sl + 5 * kWarpCols) = aux;
        }
        float cu[2][2] = {{u2.x, u2.y}, {v2.x, v2.y}};  // [plane][column]

        // ---- stages 1..T
#pragma unroll
        for (int s = 0; s < T; ++s) {
            const int n = k - s;  // arriving row (input of sweep s+1)
            float ub[2][2];       // averages of output row n-1, [plane][column]
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const float ca = cu[q][0], cb = cu[q][1];
                const float fromL = __shfl_up_sync(kFull, cb, 1);
                const float fromR = __shfl_down_sync(kFull, ca, 1);
                const float la = a_first ? ca : fromL;
                const float ra = a_last ? ca : cb;
                const float lb = ca;
                const float rb = b_last ? cb : fromR;
                const float L[2] = {la, lb}, Cc[2] = {ca, cb}, R[2] = {ra, rb};
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if constexpr (FAST) {
                        float cn = Cc[j], hn = L[j] + R[j];
                        if (n >= p.H) { cn = s0[s][q][j]; hn = s1[s][q][j]; }
                        ub[q][j] = fmaf(s2[s][q][j] + cn, we, (s3[s][q][j] + hn) * wc);
                        if (n == 0) { s2[s][q][j] = cn + hn; s3[s][q][j] = hn; }
                        else { s2[s][q][j] = s0[s][q][j] + hn; s3[s][q][j] = s1[s][q][j]; }
                        s0[s][q][j] = cn;
                        s1[s][q][j] = hn;
                    } else {
                        float l = L[j], c = Cc[j], r = R[j];
                        if (n >= p.H) { l = s2[s][q][j]; c = s3[s][q][j]; r = s4[s][q][j]; }
                        // finish the mid row with the dn taps (-1,1) (0,1) (1,1)
                        float o = s1[s][q][j];
                        o = __fadd_rn(o, __fmul_rn(wc, l));
                        o = __fadd_rn(o, __fmul_rn(we, c));
                        o = __fadd_rn(o, __fmul_rn(wc, r));
                        ub[q][j] = o;
                        // up taps (-1,-1) (0,-1) (1,-1) of the next row come from this row
                        float up = __fadd_rn(0.0f, __fmul_rn(wc, l));
                        up = __fadd_rn(up, __fmul_rn(we, c));
                        up = __fadd_rn(up, __fmul_rn(wc, r));
                        // this row becomes the mid row: its own mid taps (-1,0) (1,0); row 0
                        // takes its up taps from itself (clamp)
                        float am = (n == 0) ? up : s0[s][q][j];
                        am = __fadd_rn(am, __fmul_rn(we, l));
                        am = __fadd_rn(am, __fmul_rn(we, r));
                        s0[s][q][j] = up;
                        s1[s][q][j] = am;
                        s2[s][q][j] = l;
                        s3[s][q][j] = c;
                        s4[s][q][j] = r;
                    }
                }
            }
            // pointwise update of row n-1 with its coefficients from the ring
            int rs = kslot - (s + 1);
            if (rs < 0) rs += G::slots;
            const float *cr = ring + rs * (kPlanes * kWarpCols) + 2 * lane;
            const float2 ix2 = lds2(cr + 2 * kWarpCols), iy2 = lds2(cr + 3 * kWarpCols);
            const float2 it2 = lds2(cr + 4 * kWarpCols), ax2 = lds2(cr + 5 * kWarpCols);
            const float IX[2] = {ix2.x, ix2.y}, IY[2] = {iy2.x, iy2.y};
            const float IT[2] = {it2.x, it2.y}, AX[2] = {ax2.x, ax2.y};
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const float ubar = ub[0][j], vbar = ub[1][j];
                if constexpr (FAST) {
                    const float r = fmaf(IX[j], ubar, fmaf(IY[j], vbar, IT[j]));
                    const float t = r * AX[j];
                    cu[0][j] = fmaf(-IX[j], t, ubar);
                    cu[1][j] = fmaf(-IY[j], t, vbar);
                } else {
                    float r = __fadd_rn(__fmul_rn(IX[j], ubar), __fmul_rn(IY[j], vbar));
                    r = __fadd_rn(r, IT[j]);
                    const float t = __fdiv_rn(r, AX[j]);
                    cu[0][j] = __fsub_rn(ubar, __fmul_rn(IX[j], t));
                    cu[1][j] = __fsub_rn(vbar, __fmul_rn(IY[j], t));
                }
            }
        }

        // ---- store sweep T of row k - T
        const int r = k - T;
        if (r >= y_start && r < y_end) {
            const size_t off = (size_t)r * p.ld + xa;
            if (st_a && st_b) {
                *reinterpret_cast<float2 *>(p.u_out + off) = make_float2(cu[0][0], cu[0][1]);
                *reinterpret_cast<float2 *>(p.v_out + off) = make_float2(cu[1][0], cu[1][1]);
            } else if (st_a) {
                p.u_out[off] = cu[0][0];
                p.v_out[off] = cu[1][0];
            }
        }
        kslot = (kslot + 1 == G::slots) ? 0 : kslot + 1;
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------------------ host side

using KernelFn = void (*)(const SweepParams);

template <int T, bool FAST>
static hs_status launch_one(const SweepParams &pp, cudaStream_t stream) {
    using G = Geo<T>;
    auto fn = hs_stream_kernel<T, FAST>;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_set[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           G::smem_bytes));
        attr_set[dev] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((pp.nitems + kWarpsPerBlock - 1) / kWarpsPerBlock));
    cfg.blockDim = dim3(kWarpsPerBlock * 32);
    cfg.dynamicSmemBytes = G::smem_bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, fn, pp));
    return HS_OK;
}

static int strip_cols_for(int T) {
    switch (T) {
        case 1: return Geo<1>::strip;
        case 2: return Geo<2>::strip;
        case 3: return Geo<3>::strip;
        case 4: return Geo<4>::strip;
        case 5: return Geo<5>::strip;
        case 6: return Geo<6>::strip;
        case 7: return Geo<7>::strip;
        default: return Geo<8>::strip;
    }
}

static hs_status launch_pass(int T, bool fast, const SweepParams &pp, cudaStream_t s) {
#define HS_CASE(TT)                                                    \
    case TT: return fast ? launch_one<TT, true>(pp, s) : launch_one<TT, false>(pp, s);
    switch (T) {
        HS_CASE(1) HS_CASE(2) HS_CASE(3) HS_CASE(4) HS_CASE(5) HS_CASE(6) HS_CASE(7) HS_CASE(8)
    }
#undef HS_CASE
    HS_FAIL(HS_ERR_INVALID_ARG, "sweeps_per_pass=%d outside 1..%d", T, HS_MAX_SWEEPS_PER_PASS);
}

// Rows per work item: enough items for about one full wave of resident warps, but
// never so few rows that the 2T-row halo dominates.
static int default_seg_rows(int H, int nstrips, int T) {
    const long target = (long)sm_count() * 16;
    long nseg = (target + nstrips - 1) / nstrips;
    if (nseg < 1) nseg = 1;
    int L = (int)((H + nseg - 1) / nseg);
    L = std::max(L, 2 * T);
    L = std::max(L, 8);
    return std::min(L, H);
}

struct ResolvedConfig {
    int T;
    int seg_rows;  // 0 = derive per pass
    bool fast;
    float we, wc;
};

static hs_status resolve_config(const hs_config *cfg, ResolvedConfig *out) {
    hs_config c = {};
    if (cfg) c = *cfg;
    for (int i = 0; i < 3; ++i)
        if (c.reserved[i] != 0) HS_FAIL(HS_ERR_INVALID_ARG, "hs_config.reserved must be zero");
    out->fast = c.fast_math != 0;
    out->T = c.sweeps_per_pass > 0 ? c.sweeps_per_pass : 4;
    if (out->T > HS_MAX_SWEEPS_PER_PASS)
        HS_FAIL(HS_ERR_INVALID_ARG, "sweeps_per_pass=%d outside 1..%d", c.sweeps_per_pass,
                HS_MAX_SWEEPS_PER_PASS);
    if (c.rows_per_segment < 0) HS_FAIL(HS_ERR_INVALID_ARG, "rows_per_segment < 0");
    out->seg_rows = c.rows_per_segment;
    if (c.avg_edge == 0.0f && c.avg_corner == 0.0f) {
        out->we = kAvgEdge;
        out->wc = kAvgCorner;
    } else {
        out->we = c.avg_edge;
        out->wc = c.avg_corner;
    }
    return HS_OK;
}

static size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Runs `iters` sweeps.  State starts in (u0, v0) if `start_in_user`, else in (u1, v1);
// the final state always lands in (u0, v0).
static hs_status run_passes(const float *Ix, const float *Iy, const float *It, int H, int W,
                            int ld, float alpha2, int iters, float *u0, float *v0, float *u1,
                            float *v1, const ResolvedConfig &rc, cudaStream_t stream) {
    if (iters <= 0) return HS_OK;
    const int T = rc.T;
    const int passes = (iters + T - 1) / T;
    float *U[2] = {u0, u1}, *V[2] = {v0, v1};
    // pass i reads buffer cur and writes buffer 1 - cur; the last pass must write 0
    int cur = (passes % 2 == 0) ? 0 : 1;
    int done = 0;
    for (int i = 0; i < passes; ++i) {
        const int t = std::min(T, iters - done);
        SweepParams pp;
        pp.Ix = Ix; pp.Iy = Iy; pp.It = It;
        pp.u_in = U[cur]; pp.v_in = V[cur];
        pp.u_out = U[1 - cur]; pp.v_out = V[1 - cur];
        pp.H = H; pp.W = W; pp.ld = ld;
        pp.alpha2 = alpha2;
        pp.we = rc.we; pp.wc = rc.wc;
        const int sc = strip_cols_for(t);
        pp.nstrips = (W + sc - 1) / sc;
        pp.seg_rows = rc.seg_rows > 0 ? std::min(rc.seg_rows, H) : default_seg_rows(H, pp.nstrips, t);
        const int nseg = (H + pp.seg_rows - 1) / pp.seg_rows;
        pp.nitems = pp.nstrips * nseg;
        hs_status st = launch_pass(t, rc.fast, pp, stream);
        if (st != HS_OK) return st;
        cur = 1 - cur;
        done += t;
    }
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" {

size_t hs_sweeps_workspace_bytes(int H, int W, int ld) {
    (void)W;
    if (H < 1 || ld < 1) return 0;
    return 2 * round_up(plane_bytes(H, ld), 256);
}

size_t hs_forward_workspace_bytes(int H, int W, int ld) {
    (void)W;
    if (H < 1 || ld < 1) return 0;
    return 5 * round_up(plane_bytes(H, ld), 256);
}

hs_status hs_sweeps(const float *Ix, const float *Iy, const float *It, int H, int W, int ld,
                    float alpha2, int iters, float *u, float *v, void *workspace,
                    size_t workspace_bytes, const hs_config *cfg, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *planes[5] = {Ix, Iy, It, u, v};
    const char *names[5] = {"Ix", "Iy", "It", "u", "v"};
    for (int i = 0; i < 5; ++i)
        if ((st = check_plane(planes[i], names[i])) != HS_OK) return st;
    if (iters < 0) HS_FAIL(HS_ERR_INVALID_ARG, "iters=%d < 0", iters);
    ResolvedConfig rc;
    if ((st = resolve_config(cfg, &rc)) != HS_OK) return st;
    if (iters == 0) return HS_OK;
    const size_t need = hs_sweeps_workspace_bytes(H, W, ld);
    if (!workspace || workspace_bytes < need)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, need);
    if (!aligned16(workspace)) HS_FAIL(HS_ERR_ALIGNMENT, "workspace is not 16-byte aligned");
    const size_t pb = round_up(plane_bytes(H, ld), 256);
    float *u1 = reinterpret_cast<float *>(workspace);
    float *v1 = reinterpret_cast<float *>(reinterpret_cast<char *>(workspace) + pb);
    cudaStream_t s = (cudaStream_t)stream;
    const int passes = (iters + rc.T - 1) / rc.T;
    if (passes % 2 == 1) {
        // the state must start in the scratch pair so that the last pass ends in (u, v)
        HS_CUDA_CHECK(cudaMemcpyAsync(u1, u, plane_bytes(H, ld), cudaMemcpyDeviceToDevice, s));
        HS_CUDA_CHECK(cudaMemcpyAsync(v1, v, plane_bytes(H, ld), cudaMemcpyDeviceToDevice, s));
    }
    return run_passes(Ix, Iy, It, H, W, ld, alpha2, iters, u, v, u1, v1, rc, s);
}

hs_status hs_forward(const float *I0, const float *I1, int H, int W, int ld, float alpha,
                     int iters, float *u, float *v, void *workspace, size_t workspace_bytes,
                     const hs_config *cfg, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *planes[4] = {I0, I1, u, v};
    const char *names[4] = {"I0", "I1", "u", "v"};
    for (int i = 0; i < 4; ++i)
        if ((st = check_plane(planes[i], names[i])) != HS_OK) return st;
    if (iters < 0) HS_FAIL(HS_ERR_INVALID_ARG, "iters=%d < 0", iters);
    ResolvedConfig rc;
    if ((st = resolve_config(cfg, &rc)) != HS_OK) return st;
    const size_t need = hs_forward_workspace_bytes(H, W, ld);
    if (!workspace || workspace_bytes < need)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, need);
    if (!aligned16(workspace)) HS_FAIL(HS_ERR_ALIGNMENT, "workspace is not 16-byte aligned");
    const size_t pb = round_up(plane_bytes(H, ld), 256);
    char *w = reinterpret_cast<char *>(workspace);
    float *Ix = reinterpret_cast<float *>(w);
    float *Iy = reinterpret_cast<float *>(w + pb);
    float *It = reinterpret_cast<float *>(w + 2 * pb);
    float *u1 = reinterpret_cast<float *>(w + 3 * pb);
    float *v1 = reinterpret_cast<float *>(w + 4 * pb);
    cudaStream_t s = (cudaStream_t)stream;
    if ((st = hs_derivs(I0, I1, H, W, ld, Ix, Iy, It, stream)) != HS_OK) return st;
    const int passes = iters > 0 ? (iters + rc.T - 1) / rc.T : 0;
    // zero the buffer pair the first pass reads (u, v themselves when no pass runs)
    float *zu = (passes % 2 == 1) ? u1 : u;
    float *zv = (passes % 2 == 1) ? v1 : v;
    HS_CUDA_CHECK(cudaMemsetAsync(zu, 0, plane_bytes(H, ld), s));
    HS_CUDA_CHECK(cudaMemsetAsync(zv, 0, plane_bytes(H, ld), s));
    const float alpha2 = alpha * alpha;  // one FP32 rounding, as the program's ScalarOp
    return run_passes(Ix, Iy, It, H, W, ld, alpha2, iters, u, v, u1, v1, rc, s);
}

}  // extern "C"
