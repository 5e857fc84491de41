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

constexpr int kWarpCols = 64;                 // columns per strip (2 per lane)
constexpr int kPrefetch = 3;                  // rows in flight per warp
constexpr int kRawSlots = kPrefetch + 1;      // raw-row ring depth (a power of two)
constexpr int kRawPlanes = 5;                 // u, v, Ix, Iy, It as copied from HBM
constexpr int kWarpsPerBlock = 4;             // independent warps per CTA
constexpr unsigned kFull = 0xffffffffu;

template <int T>
struct Geo {
    static constexpr int halo = (T + 1) & ~1;                  // even, so lanes load float2
    static constexpr int strip = kWarpCols - 2 * halo;         // output columns per strip
    static constexpr int coef_slots = T + 1;                   // rows k-T .. k
    static constexpr int raw_floats = kRawSlots * kRawPlanes * kWarpCols;
    static constexpr int coef_floats = coef_slots * 2 * 32 * 4;  // [slot][column][lane] float4
    static constexpr int warp_floats = raw_floats + coef_floats;
    static constexpr int smem_bytes = kWarpsPerBlock * warp_floats * (int)sizeof(float);
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

// Hardware reciprocal approximation (PTX rcp.approx, about 1 ulp) for the fast form.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }

// Sliding three-row window of one stage, one plane, one column.
//   fast : with Y(k) = we*c(k) + wc*h(k) (h = left + right), the average of row n-1 is
//          Y(n-2) + we*h(n-1) + Y(n).  Z = Y(n-2) + we*h(n-1) and Y1 = Y(n-1) are kept,
//          so a row costs 5 operations and 2 registers.
//   exact: A0 = next row's accumulator holding its up taps (taken from row n-1),
//          A1 = row n-1's accumulator holding its up and mid taps, l1/c1/r1 = row n-1
//          (read only for the bottom clamp)
template <bool FAST>
struct Win;
template <>
struct Win<true> {
    float Z, Y1;
};
template <>
struct Win<false> {
    float A0, A1, l1, c1, r1;
};

// Row n arrives (values l, c, r at this column); returns the average of row n-1 and
// advances the window.  EDGE: the row may be row 0 (top clamp) or past the bottom
// (replaced by row H-1, the bottom clamp).
template <bool EDGE>
__device__ __forceinline__ float win_step(Win<true> &w, float l, float c, float r, int n, int H,
                                          float we, float wc) {
    const float hn = l + r;
    float yn = fmaf(we, c, wc * hn);
    if (EDGE && n >= H) yn = w.Y1;  // the row below H-1 is row H-1
    const float out = w.Z + yn;
    w.Z = fmaf(we, hn, (EDGE && n == 0) ? yn : w.Y1);  // row 0's up row is row 0
    w.Y1 = yn;
    return out;
}

template <bool EDGE>
__device__ __forceinline__ float win_step(Win<false> &w, float l, float c, float r, int n, int H,
                                          float we, float wc) {
    if (EDGE && n >= H) { l = w.l1; c = w.c1; r = w.r1; }
    // taps in row-major order: (-1,-1) (0,-1) (1,-1) | (-1,0) (1,0) | (-1,1) (0,1) (1,1)
    float o = w.A1;                              // row n-1: up and mid taps done
    o = __fadd_rn(o, __fmul_rn(wc, l));          // its dn taps come from row n
    o = __fadd_rn(o, __fmul_rn(we, c));
    o = __fadd_rn(o, __fmul_rn(wc, r));
    float up = __fadd_rn(0.0f, __fmul_rn(wc, l));  // row n+1's up taps come from row n
    up = __fadd_rn(up, __fmul_rn(we, c));
    up = __fadd_rn(up, __fmul_rn(wc, r));
    float am = (EDGE && n == 0) ? up : w.A0;     // row 0's up taps are its own (clamp)
    am = __fadd_rn(am, __fmul_rn(we, l));        // row n's mid taps
    am = __fadd_rn(am, __fmul_rn(we, r));
    w.A0 = up;
    w.A1 = am;
    if (EDGE) { w.l1 = l; w.c1 = c; w.r1 = r; }
    return o;
}

// Per-warp context of one work item.
struct Item {
    float *raw;    // [kRawSlots][kRawPlanes][64] floats
    float4 *coef;  // [T+1][2][32]
    int lane, lc;
    bool a_first, a_last, b_last, st_a, st_b;
    int xa, y_start, y_end;
};

__device__ __forceinline__ void issue_row(const Item &it, int slot, int row, const SweepParams &p) {
    row = min(max(row, 0), p.H - 1);
    const size_t off = (size_t)row * p.ld + it.lc;
    float *base = it.raw + slot * (kRawPlanes * kWarpCols) + 2 * it.lane;
    cp_async8(base + 0 * kWarpCols, p.u_in + off);
    cp_async8(base + 1 * kWarpCols, p.v_in + off);
    cp_async8(base + 2 * kWarpCols, p.Ix + off);
    cp_async8(base + 3 * kWarpCols, p.Iy + off);
    cp_async8(base + 4 * kWarpCols, p.It + off);
    cp_async_commit();
}

// One streaming step: row k arrives at stage 0, stage s emits sweep s+1 of row k-s-1.
template <int T, bool FAST, bool XEDGE, bool EDGE>
__device__ __forceinline__ void stream_step(const SweepParams &p, const Item &it, Win<FAST> (&w)[T][2][2],
                                            int k, int rslot, int cslot) {
    // prefetch row k + kPrefetch into the slot row k-1 used, then wait for row k
    issue_row(it, (rslot + kPrefetch) & (kRawSlots - 1), k + kPrefetch, p);
    cp_async_wait<kPrefetch>();

    // stage 0: unpack row k; pack its coefficients with the denominator term
    const float *raw = it.raw + rslot * (kRawPlanes * kWarpCols) + 2 * it.lane;
    const float2 u2 = lds2(raw), v2 = lds2(raw + kWarpCols);
    {
        const float2 ix = lds2(raw + 2 * kWarpCols), iy = lds2(raw + 3 * kWarpCols);
        const float2 t2 = lds2(raw + 4 * kWarpCols);
        float ax, ay;
        if constexpr (FAST) {
            ax = rcp_approx(fmaf(iy.x, iy.x, fmaf(ix.x, ix.x, p.alpha2)));
            ay = rcp_approx(fmaf(iy.y, iy.y, fmaf(ix.y, ix.y, p.alpha2)));
        } else {
            ax = __fadd_rn(__fadd_rn(p.alpha2, __fmul_rn(ix.x, ix.x)), __fmul_rn(iy.x, iy.x));
            ay = __fadd_rn(__fadd_rn(p.alpha2, __fmul_rn(ix.y, ix.y)), __fmul_rn(iy.y, iy.y));
        }
        float4 *cs = it.coef + cslot * 64 + it.lane;
        cs[0] = make_float4(ix.x, iy.x, t2.x, ax);
        cs[32] = make_float4(ix.y, iy.y, t2.y, ay);
    }
    float cu[2][2] = {{u2.x, u2.y}, {v2.x, v2.y}};  // [plane][column]

#pragma unroll
    for (int s = 0; s < T; ++s) {
        const int n = k - s;  // arriving row (input of sweep s+1)
        float ub[2][2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float ca = cu[q][0], cb = cu[q][1];
            const float fromL = __shfl_up_sync(kFull, cb, 1);
            const float fromR = __shfl_down_sync(kFull, ca, 1);
            float la = fromL, ra = cb, rb = fromR;
            if constexpr (XEDGE) {
                la = it.a_first ? ca : la;
                ra = it.a_last ? ca : ra;
                rb = it.b_last ? cb : rb;
            }
            ub[q][0] = win_step<EDGE>(w[s][q][0], la, ca, ra, n, p.H, p.we, p.wc);
            ub[q][1] = win_step<EDGE>(w[s][q][1], ca, cb, rb, n, p.H, p.we, p.wc);
        }
        // pointwise update of row n-1 with its coefficients
        int rs = cslot - (s + 1);
        if (rs < 0) rs += Geo<T>::coef_slots;
        const float4 *cr = it.coef + rs * 64 + it.lane;
        const float4 C[2] = {cr[0], cr[32]};
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float ubar = ub[0][j], vbar = ub[1][j];
            if constexpr (FAST) {
                const float r = fmaf(C[j].x, ubar, fmaf(C[j].y, vbar, C[j].z));
                const float t = r * C[j].w;
                cu[0][j] = fmaf(-C[j].x, t, ubar);
                cu[1][j] = fmaf(-C[j].y, t, vbar);
            } else {
                float r = __fadd_rn(__fmul_rn(C[j].x, ubar), __fmul_rn(C[j].y, vbar));
                r = __fadd_rn(r, C[j].z);
                const float t = __fdiv_rn(r, C[j].w);
                cu[0][j] = __fsub_rn(ubar, __fmul_rn(C[j].x, t));
                cu[1][j] = __fsub_rn(vbar, __fmul_rn(C[j].y, t));
            }
        }
    }

    // store sweep T of row k - T
    const int r = k - T;
    if (r >= it.y_start && r < it.y_end) {
        const size_t off = (size_t)r * p.ld + it.xa;
        if (it.st_a && it.st_b) {
            *reinterpret_cast<float2 *>(p.u_out + off) = make_float2(cu[0][0], cu[0][1]);
            *reinterpret_cast<float2 *>(p.v_out + off) = make_float2(cu[1][0], cu[1][1]);
        } else if (it.st_a) {
            p.u_out[off] = cu[0][0];
            p.v_out[off] = cu[1][0];
        }
    }
}

template <int T, bool FAST, bool XEDGE>
__device__ __forceinline__ void stream_item(const SweepParams &p, const Item &it) {
    const int k0 = max(0, it.y_start - T);
    const int k_end = it.y_end - 1 + T;
    Win<FAST> w[T][2][2];
#pragma unroll
    for (int s = 0; s < T; ++s)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int j = 0; j < 2; ++j) w[s][q][j] = Win<FAST>{};

#pragma unroll
    for (int i = 0; i < kPrefetch; ++i) issue_row(it, i, k0 + i, p);

    // Steps in [klo, khi] have no stage at row 0 or past row H-2: no clamp logic.
    const int klo = max(k0, T);
    const int khi = min(k_end, p.H - 2);
    int k = k0, rslot = 0, cslot = 0;
    auto advance = [&]() {
        ++k;
        rslot = (rslot + 1) & (kRawSlots - 1);
        cslot = (cslot + 1 == Geo<T>::coef_slots) ? 0 : cslot + 1;
    };
    if (klo + 1 <= khi) {
        for (; k < klo; advance()) stream_step<T, FAST, XEDGE, true>(p, it, w, k, rslot, cslot);
        while (k + 1 <= khi) {
            stream_step<T, FAST, XEDGE, false>(p, it, w, k, rslot, cslot);
            advance();
            stream_step<T, FAST, XEDGE, false>(p, it, w, k, rslot, cslot);
            advance();
        }
        // Here k <= H-1, so row H-1 reaches every stage in the tail loop below.  The
        // bottom-clamp values are written and read only there; dropping the head loop's
        // copies keeps them out of the main loop's live registers.
        if constexpr (!FAST) {
#pragma unroll
            for (int s = 0; s < T; ++s)
#pragma unroll
                for (int q = 0; q < 2; ++q)
#pragma unroll
                    for (int j = 0; j < 2; ++j) w[s][q][j].l1 = w[s][q][j].c1 = w[s][q][j].r1 = 0.f;
        }
    }
    for (; k <= k_end; advance()) stream_step<T, FAST, XEDGE, true>(p, it, w, k, rslot, cslot);
    cp_async_wait<0>();
}

// Resident CTAs per SM the register budget is sized for (shared memory allows it too).
// (Measured: capping registers for more CTAs costs more ILP than it gains.)
constexpr int min_blocks(int T) { return T <= 4 ? 4 : (T <= 6 ? 3 : 2); }

template <int T, bool FAST>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, min_blocks(T))
    hs_stream_kernel(const SweepParams p) {
    using G = Geo<T>;
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *wbase = reinterpret_cast<float *>(smem4) + warp * G::warp_floats;

    griddep_launch_dependents();
    griddep_wait();

    const int item = blockIdx.x * kWarpsPerBlock + warp;
    if (item >= p.nitems) return;  // warp-uniform
    const int strip = item % p.nstrips;
    const int seg = item / p.nstrips;
    const int x0 = strip * G::strip - G::halo;
    Item it;
    it.raw = wbase;
    it.coef = reinterpret_cast<float4 *>(wbase + G::raw_floats);
    it.lane = lane;
    it.xa = x0 + 2 * lane;
    const int xb = it.xa + 1;
    // Column pair each lane loads: its own when it starts inside the image (xa is even
    // and ld is a multiple of 4, so xa + 1 < ld), any in-bounds pair otherwise -- columns
    // outside the image never feed a stored pixel.
    it.lc = (it.xa >= 0 && it.xa < p.W) ? it.xa : 0;
    it.a_first = (it.xa == 0);
    it.a_last = (it.xa == p.W - 1);
    it.b_last = (xb == p.W - 1);
    const int vlo = strip * G::strip, vhi = min(vlo + G::strip, p.W);
    it.st_a = (it.xa >= vlo && it.xa < vhi);
    it.st_b = (xb >= vlo && xb < vhi);
    it.y_start = seg * p.seg_rows;
    it.y_end = min(p.H, it.y_start + p.seg_rows);
    // only strips reaching an image side need the horizontal clamp selects
    if (x0 <= 0 || x0 + kWarpCols >= p.W) stream_item<T, FAST, true>(p, it);
    else stream_item<T, FAST, false>(p, it);
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
