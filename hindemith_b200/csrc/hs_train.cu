// hs_train.cu -- batched differentiable Horn-Schunck: forward with checkpoints and the
// temporally blocked adjoint, for n pairs per launch.
//
// Forward.  The sweeps run interval by interval (ckpt_every sweeps each): every pass is
// one table-driven launch over all pairs; an interval's first pass reads checkpoint b and
// its last pass writes checkpoint b+1, so checkpoints cost no copies.
//
// Backward, interval by interval in reverse:
//  1. Recompute the interval's states x_{k+1} with "dump" passes of the forward kernel:
//     every stage of a pass also writes its sweep, so T states cost one pass.
//  2. Adjoint passes of TB sweeps each.  Because the clamp-to-edge average is symmetric
//     in each axis, its transpose is itself (A^T = A), so the adjoint of a sweep is
//     "pointwise map M, then A": with lambda = dL/dx_{k+1},
//         g = Ix lu + Iy lv, lr = -g/d, z = lambda + lr (Ix, Iy), lambda_k = A z,
//     and the gradient accumulations of sweep k need ubar, vbar, t of sweep k, which follow
//     pointwise from x_{k+1}:  t = (Ix u_{k+1} + Iy v_{k+1} + It) / alpha^2,
//     ubar = u_{k+1} + Ix t, vbar = v_{k+1} + Iy t  (d t = r and r - (Ix^2+Iy^2) t = alpha^2 t).
//     The adjoint pass is therefore the forward's register pipeline with M in place of
//     the Jacobi update: stage 0 applies M to the incoming lambda row, stage s applies A
//     and then M of the next sweep; per-row accumulators live in a shared-memory ring
//     beside the coefficients and are added to HBM once per pass.
//  3. Transposed derivative stencils and the alpha reduction, per pair.
// The gradient needs alpha != 0 (t is recovered through 1/alpha^2).
#include <algorithm>
#include <mutex>
#include <vector>

#include "hs_stream4.cuh"

namespace hs {

constexpr int kMaxTrainPairs = 32;
constexpr int kMaxTB = 5;
constexpr int kAdjMaxDepth = 4;     // deepest adjoint pass the backward plans
constexpr int kAdjItemsPerSmMax = 16;  // adjoint work items (warps) per SM and launch, at most
constexpr int kMinStripCols = 52;   // narrowest adjoint strip (depth <= 5): 64 less 6 each side
// Warps per CTA of the backward's launches.  Its recompute (dump) passes and adjoint passes
// run on two streams at once; with 4-warp CTAs each SM holds blocks of one kind, while one-warp
// CTAs interleave the two kinds warp by warp on every SM (measured on B200, 16 x 512^2, 200
// sweeps: forward + backward 9.1 ms against 10.2 ms with one-warp dump passes).  The forward's
// passes run alone and use one-warp CTAs (kPassWarps).
constexpr int kBackwardWarps = 4;

// ------------------------------------------------------------------ table-driven pass

struct PassTable {
    SweepParams pair[kMaxTrainPairs];
    int item_prefix[kMaxTrainPairs + 1];
    int npairs;
    bool wide;  // 4 columns per lane (fast form; every pair of the table)
};

__device__ __forceinline__ int find_pair(const int *prefix, int n, int item) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int T, bool FAST, int WP>
__global__ void __launch_bounds__(WP * 32, (T <= 4 ? 16 : (T <= 6 ? 12 : 8)) / WP)
    hs_table_pass_kernel(const __grid_constant__ PassTable tab) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *wbase = reinterpret_cast<float *>(smem4) + warp * Geo<T>::warp_floats;
    griddep_launch_dependents();
    griddep_wait();
    const int item = blockIdx.x * WP + warp;
    if (item >= tab.item_prefix[tab.npairs]) return;
    const int pi = find_pair(tab.item_prefix, tab.npairs, item);
    const SweepParams &p = tab.pair[pi];
    const int local = item - tab.item_prefix[pi];
    Item it;
    init_item<T>(it, p, local % p.nstrips, local / p.nstrips, lane, wbase);
    if (p.dump) run_item<T, FAST, true>(p, it);
    else run_item<T, FAST, false>(p, it);
}

template <int T, bool FAST, int WP>
static hs_status launch_table_wp(const PassTable &tab, cudaStream_t s) {
    auto fn = hs_table_pass_kernel<T, FAST, WP>;
    static bool attr[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           WP * Geo<T>::warp_floats * (int)sizeof(float)));
        attr[dev] = true;
    }
    const int items = tab.item_prefix[tab.npairs];
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((items + WP - 1) / WP));
    cfg.blockDim = dim3(WP * 32);
    cfg.dynamicSmemBytes = WP * Geo<T>::warp_floats * (int)sizeof(float);
    cfg.stream = s;
    cudaLaunchAttribute a[1];
    a[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    a[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = a;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, fn, tab));
    return HS_OK;
}

// The same pass in the 4-columns-per-lane layout (fast form only).
template <int T, int WP>
__global__ void __launch_bounds__(WP * 32, (T <= 4 ? 12 : 8) / WP)
    hs_table_pass_w_kernel(const __grid_constant__ PassTable tab) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *wbase = reinterpret_cast<float *>(smem4) + warp * GeoW<T>::warp_floats;
    griddep_launch_dependents();
    griddep_wait();
    const int item = blockIdx.x * WP + warp;
    if (item >= tab.item_prefix[tab.npairs]) return;
    const int pi = find_pair(tab.item_prefix, tab.npairs, item);
    const SweepParams &p = tab.pair[pi];
    const int local = item - tab.item_prefix[pi];
    ItemW it;
    init_item_w<T>(it, p, local % p.nstrips, local / p.nstrips, lane, wbase);
    if (p.dump) run_item_w<T, true>(p, it);
    else run_item_w<T, false>(p, it);
}

template <int T, int WP>
static hs_status launch_table_w_wp(const PassTable &tab, cudaStream_t s) {
    auto fn = hs_table_pass_w_kernel<T, WP>;
    static bool attr[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           WP * GeoW<T>::warp_floats * (int)sizeof(float)));
        attr[dev] = true;
    }
    const int items = tab.item_prefix[tab.npairs];
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((items + WP - 1) / WP));
    cfg.blockDim = dim3(WP * 32);
    cfg.dynamicSmemBytes = WP * GeoW<T>::warp_floats * (int)sizeof(float);
    cfg.stream = s;
    cudaLaunchAttribute a[1];
    a[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    a[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = a;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, fn, tab));
    return HS_OK;
}

// The forward's passes in one-warp CTAs, the backward's recompute passes (depth <= 5, every
// pair of a table dumps or none does) in kBackwardWarps.
constexpr int kMaxDumpDepth = 5;
template <int T, bool FAST>
static hs_status launch_table(const PassTable &tab, cudaStream_t s) {
    if (!tab.pair[0].dump) return launch_table_wp<T, FAST, kPassWarps>(tab, s);
    if constexpr (T <= kMaxDumpDepth) return launch_table_wp<T, FAST, kBackwardWarps>(tab, s);
    else HS_FAIL(HS_ERR_INVALID_ARG, "recompute pass depth %d above %d", T, kMaxDumpDepth);
}
template <int T>
static hs_status launch_table_w(const PassTable &tab, cudaStream_t s) {
    if (!tab.pair[0].dump) return launch_table_w_wp<T, kPassWarps>(tab, s);
    if constexpr (T <= kMaxDumpDepth) return launch_table_w_wp<T, kBackwardWarps>(tab, s);
    else HS_FAIL(HS_ERR_INVALID_ARG, "recompute pass depth %d above %d", T, kMaxDumpDepth);
}

static hs_status launch_table_any(int T, bool fast, const PassTable &tab, cudaStream_t s) {
    if (tab.wide) {
        switch (T) {
            case 1: return launch_table_w<1>(tab, s);
            case 2: return launch_table_w<2>(tab, s);
            case 3: return launch_table_w<3>(tab, s);
            case 4: return launch_table_w<4>(tab, s);
            case 5: return launch_table_w<5>(tab, s);
            case 6: return launch_table_w<6>(tab, s);
            case 7: return launch_table_w<7>(tab, s);
            case 8: return launch_table_w<8>(tab, s);
        }
        HS_FAIL(HS_ERR_INVALID_ARG, "pass depth %d outside 1..8", T);
    }
#define HS_CASE(TT) \
    case TT: return fast ? launch_table<TT, true>(tab, s) : launch_table<TT, false>(tab, s);
    switch (T) { HS_CASE(1) HS_CASE(2) HS_CASE(3) HS_CASE(4) HS_CASE(5) HS_CASE(6) HS_CASE(7) HS_CASE(8) }
#undef HS_CASE
    HS_FAIL(HS_ERR_INVALID_ARG, "pass depth %d outside 1..8", T);
}

// ------------------------------------------------------------------ adjoint pass

struct AdjPair {
    const float *Ix, *Iy, *It;
    const float *lu_in, *lv_in;
    float *lu_out, *lv_out;
    const float *xu[kMaxTB], *xv[kMaxTB];  // x_{k_hi - s}, s = 0..TB-1
    float *aIx, *aIy, *aIt;                // accumulators (+=, one owner per pixel per launch)
    double *a2part;                        // per-item partial sums of dL/dalpha^2 (+=)
    const float *alpha_dev;
    int H, W, ld, seg_rows, nstrips;
};

struct AdjTable {
    AdjPair pair[kMaxTrainPairs];
    int item_prefix[kMaxTrainPairs + 1];
    int npairs;
    float we, wc;
};

template <int TB>
struct AdjGeo {
    static constexpr int coef_slots = TB + 1;
    static constexpr int raw_floats = Geo<TB>::raw_floats;
    static constexpr int ring_floats = coef_slots * 2 * 2 * 32 * 4;  // [slot][4][lane] float4 pairs
    static constexpr int warp_floats = raw_floats + ring_floats;
    static constexpr int smem_bytes = kBackwardWarps * warp_floats * (int)sizeof(float);
};

// M of one sweep at one column: lambda (lu, lv) -> z, adding this sweep's gradient terms to
// the accumulators (aIx, aIy, aIt, aA2); (xu, xv) = x_{k+1}, d the denominator.
// With g = Ix lu + Iy lv, lr = -g/d, t = (Ix xu + Iy xv + It)/alpha^2 and z = lambda + lr (Ix, Iy):
//   dIx += -lu t + lr ubar + 2 Ix (g t / d) = lr xu - t zu   (ubar = xu + Ix t, g t / d = -lr t)
//   dIy += lr xv - t zv,   dIt += lr,   dalpha^2 += -lr t
// The lane's two columns run as packed pairs.  The ring holds, per pair,
// (Ix, Iy), (It, -1/d), (aIx, aIy) and (aIt, aA2); nia2 = -1/alpha^2.  With the negated
// factors: lr = g (-1/d), -t = (Ix xu + Iy xv + It)(-1/alpha^2), dIx += lr xu + (-t) zu,
// dalpha^2 += lr (-t).
__device__ __forceinline__ void adj_point2(float2 lu, float2 lv, float4 CA, float4 CB, float2 xu,
                                           float2 xv, float2 nia2, float2 &zu, float2 &zv,
                                           float4 &AA, float4 &AB) {
    const float2 cx = make_float2(CA.x, CA.y), cy = make_float2(CA.z, CA.w);
    const float2 ct = make_float2(CB.x, CB.y), nw = make_float2(CB.z, CB.w);
    const float2 g = fma2(cx, lu, mul2(cy, lv));
    const float2 lr = mul2(g, nw);
    zu = fma2(lr, cx, lu);
    zv = fma2(lr, cy, lv);
    const float2 nt = mul2(fma2(cx, xu, fma2(cy, xv, ct)), nia2);
    const float2 aIx = fma2(nt, zu, fma2(lr, xu, make_float2(AA.x, AA.y)));
    const float2 aIy = fma2(nt, zv, fma2(lr, xv, make_float2(AA.z, AA.w)));
    const float2 aIt = add2(make_float2(AB.x, AB.y), lr);
    const float2 aA = fma2(lr, nt, make_float2(AB.z, AB.w));
    AA = make_float4(aIx.x, aIx.y, aIy.x, aIy.y);
    AB = make_float4(aIt.x, aIt.y, aA.x, aA.y);
}

__device__ __forceinline__ void prefetch_l2(const float *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Global loads one step ahead: the state rows every stage uses at step k; and an L2
// prefetch of the rows of step k + kAdjL2Ahead, so that the register loads find them in L2
// (the loads' latency was the adjoint's leading stall).
constexpr int kAdjL2Ahead = 2;
template <int TB>
__device__ __forceinline__ void adj_prefetch(const AdjPair &P, const Item &it, int k,
                                             float2 (&xs)[TB][2]) {
#pragma unroll
    for (int s = 0; s < TB; ++s) {
        const int r = min(max(k - s, 0), P.H - 1);
        const size_t off = (size_t)r * P.ld + it.lc2;
        xs[s][0] = __ldg(reinterpret_cast<const float2 *>(P.xu[s] + off));
        xs[s][1] = __ldg(reinterpret_cast<const float2 *>(P.xv[s] + off));
        const int r2 = min(max(k + kAdjL2Ahead - s, 0), P.H - 1);
        const size_t off2 = (size_t)r2 * P.ld + it.lc2;
        prefetch_l2(P.xu[s] + off2);
        prefetch_l2(P.xv[s] + off2);
    }
}

template <int TB, bool XEDGE, bool EDGE>
__device__ __forceinline__ void adj_step(const AdjPair &P, const SweepParams &lp, const Item &it,
                                         float4 *ring, Win<true> (&w)[TB][2], float inv_a2,
                                         float we, float wc, int k, int rslot, int cslot,
                                         float2 (&xs)[TB][2], float &a2s) {
    __syncwarp();
    issue_row<TB>(it, (rslot + kPrefetch) & (kRawSlots - 1), min(k + kPrefetch, it.y_end - 1 + TB), lp);
    cp_async_wait<kPrefetch>();
    __syncwarp();

    // stage 0: lambda row k arrives; coefficients, zeroed accumulators, then M
    constexpr int RW = Geo<TB>::rw;
    const float *raw = it.raw + rslot * (kRawPlanes * RW) + Geo<TB>::sh + 2 * it.lane;
    const float2 l2u = lds2(raw), l2v = lds2(raw + RW);
    float2 cu[2];  // [plane]: the lane's column pair
    const float2 nia2 = f2(-inv_a2, -inv_a2);
    {
        const float2 ix = lds2(raw + 2 * RW), iy = lds2(raw + 3 * RW);
        const float2 t2 = lds2(raw + 4 * RW);
        const float nax = -rcp_approx(fmaf(iy.x, iy.x, fmaf(ix.x, ix.x, it.alpha2)));
        const float nay = -rcp_approx(fmaf(iy.y, iy.y, fmaf(ix.y, ix.y, it.alpha2)));
        const float4 CA = make_float4(ix.x, ix.y, iy.x, iy.y), CB = make_float4(t2.x, t2.y, nax, nay);
        float4 *slot = ring + cslot * 128 + it.lane;
        float4 AA = make_float4(0.f, 0.f, 0.f, 0.f), AB = AA;
        adj_point2(l2u, l2v, CA, CB, xs[0][0], xs[0][1], nia2, cu[0], cu[1], AA, AB);
        slot[0] = CA;
        slot[32] = CB;
        slot[64] = AA;
        slot[96] = AB;
    }
#pragma unroll
    for (int s = 1; s <= TB; ++s) {
        const int n = k - s + 1;  // arriving row
        float2 lam[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float2 c = cu[q];
            const float fromL = __shfl_up_sync(kFull, c.y, 1);
            const float fromR = __shfl_down_sync(kFull, c.x, 1);
            // (the packed left + right measured faster here than the forward's scalar sums)
            float2 l = f2(fromL, c.x), r = f2(c.y, fromR);
            if constexpr (XEDGE) {
                l.x = it.a_first ? c.x : l.x;
                r.x = it.a_last ? c.x : r.x;
                r.y = it.b_last ? c.y : r.y;
            }
            lam[q] = win_step_h<EDGE>(w[s - 1][q], add2(l, r), c, n, P.H, f2(we, we), f2(wc, wc));
        }
        if (s < TB) {  // M of the next sweep at row k - s
            int rs = cslot - s;
            if (rs < 0) rs += AdjGeo<TB>::coef_slots;
            float4 *slot = ring + rs * 128 + it.lane;
            float4 AA = slot[64], AB = slot[96];
            adj_point2(lam[0], lam[1], slot[0], slot[32], xs[s][0], xs[s][1], nia2, cu[0], cu[1], AA, AB);
            slot[64] = AA;
            slot[96] = AB;
        } else {
            cu[0] = lam[0];
            cu[1] = lam[1];
        }
    }

    // flush the accumulators of row k - (TB-1): its last sweep's M ran in this step.  The
    // adds are reductions performed in L2 (no value comes back to the warp); each pixel has
    // one owner per launch and launches are stream-ordered, so the sums are deterministic.
    {
        const int r = k - (TB - 1);
        if (r >= it.y_start && r < it.y_end) {
            int rs = cslot - (TB - 1);
            if (rs < 0) rs += AdjGeo<TB>::coef_slots;
            const float4 *slot = ring + rs * 128 + it.lane;
            const float4 AA = slot[64], AB = slot[96];  // (aIx, aIy) and (aIt, aA2) pairs
            const size_t off = (size_t)r * P.ld + it.xa;
            if (it.st_a && it.st_b) {
                atomicAdd(reinterpret_cast<float2 *>(P.aIx + off), make_float2(AA.x, AA.y));
                atomicAdd(reinterpret_cast<float2 *>(P.aIy + off), make_float2(AA.z, AA.w));
                atomicAdd(reinterpret_cast<float2 *>(P.aIt + off), make_float2(AB.x, AB.y));
                a2s += AB.z + AB.w;
            } else if (it.st_a) {
                atomicAdd(P.aIx + off, AA.x);
                atomicAdd(P.aIy + off, AA.z);
                atomicAdd(P.aIt + off, AB.x);
                a2s += AB.z;
            }
        }
    }
    adj_prefetch<TB>(P, it, k + 1, xs);  // for the next step
    // store lambda_{k_hi - TB} of row k - TB
    {
        const int r = k - TB;
        if (r >= it.y_start && r < it.y_end) {
            const size_t off = (size_t)r * P.ld + it.xa;
            if (it.st_a && it.st_b) {
                *reinterpret_cast<float2 *>(P.lu_out + off) = cu[0];
                *reinterpret_cast<float2 *>(P.lv_out + off) = cu[1];
            } else if (it.st_a) {
                P.lu_out[off] = cu[0].x;
                P.lv_out[off] = cu[1].x;
            }
        }
    }
}

template <int TB, bool XEDGE>
__device__ __forceinline__ void adj_item(const AdjPair &P, const SweepParams &lp, const Item &it,
                                         float4 *ring, float we, float wc, int local) {
    const float a = __ldg(P.alpha_dev);
    const float inv_a2 = 1.0f / (a * a);
    const int k0 = max(0, it.y_start - TB);
    const int k_end = it.y_end - 1 + TB;
    Win<true> w[TB][2];
#pragma unroll
    for (int s = 0; s < TB; ++s)
#pragma unroll
        for (int q = 0; q < 2; ++q) w[s][q] = Win<true>{};
#pragma unroll
    for (int i = 0; i < kPrefetch; ++i) issue_row<TB>(it, i, k0 + i, lp);
    float2 xs[TB][2];
    float a2s = 0.f;
    adj_prefetch<TB>(P, it, k0, xs);
    const int klo = max(k0, TB);
    const int khi = min(k_end, P.H - 2);
    int k = k0, rslot = 0, cslot = 0;
    auto advance = [&]() {
        ++k;
        rslot = (rslot + 1) & (kRawSlots - 1);
        cslot = (cslot + 1 == AdjGeo<TB>::coef_slots) ? 0 : cslot + 1;
    };
    if (klo + 1 <= khi) {
        for (; k < klo; advance()) adj_step<TB, XEDGE, true>(P, lp, it, ring, w, inv_a2, we, wc, k, rslot, cslot, xs, a2s);
        while (k + 1 <= khi) {
            adj_step<TB, XEDGE, false>(P, lp, it, ring, w, inv_a2, we, wc, k, rslot, cslot, xs, a2s);
            advance();
            adj_step<TB, XEDGE, false>(P, lp, it, ring, w, inv_a2, we, wc, k, rslot, cslot, xs, a2s);
            advance();
        }
    }
    for (; k <= k_end; advance()) adj_step<TB, XEDGE, true>(P, lp, it, ring, w, inv_a2, we, wc, k, rslot, cslot, xs, a2s);
    cp_async_wait<0>();
    // this item's share of dL/dalpha^2: fixed-order butterfly, one owner per slot per launch
    double d = (double)a2s;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(kFull, d, o);
    if (it.lane == 0) P.a2part[local] += d;
}

// resident warps per SM the register budget is sized for: depth <= 3 fits 16
constexpr int adj_res_warps(int TB) { return TB <= 3 ? 16 : 12; }

template <int TB>
__global__ void __launch_bounds__(kBackwardWarps * 32, adj_res_warps(TB) / kBackwardWarps)
    hs_adjoint_pass_kernel(const __grid_constant__ AdjTable tab) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *wbase = reinterpret_cast<float *>(smem4) + warp * AdjGeo<TB>::warp_floats;
    griddep_launch_dependents();
    griddep_wait();
    const int item = blockIdx.x * kBackwardWarps + warp;
    if (item >= tab.item_prefix[tab.npairs]) return;
    const int pi = find_pair(tab.item_prefix, tab.npairs, item);
    const AdjPair &P = tab.pair[pi];
    const int local = item - tab.item_prefix[pi];
    // the row loads of the streaming machinery read lambda where the forward reads (u, v)
    SweepParams lp;
    lp.Ix = P.Ix;
    lp.Iy = P.Iy;
    lp.It = P.It;
    lp.u_in = P.lu_in;
    lp.v_in = P.lv_in;
    lp.H = P.H;
    lp.W = P.W;
    lp.ld = P.ld;
    lp.seg_rows = P.seg_rows;
    lp.nstrips = P.nstrips;
    lp.alpha2 = 0.f;
    lp.alpha_dev = P.alpha_dev;
    lp.dump = 0;
    Item it;
    init_item<TB>(it, lp, local % P.nstrips, local / P.nstrips, lane, wbase);
    it.coef = reinterpret_cast<float4 *>(wbase + AdjGeo<TB>::raw_floats);
    const int x0 = it.xa - 2 * lane;
    if (x0 <= 0 || x0 + kWarpCols >= P.W) adj_item<TB, true>(P, lp, it, it.coef, tab.we, tab.wc, local);
    else adj_item<TB, false>(P, lp, it, it.coef, tab.we, tab.wc, local);
}

template <int TB>
static hs_status launch_adj(const AdjTable &tab, cudaStream_t s) {
    auto fn = hs_adjoint_pass_kernel<TB>;
    static bool attr[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, AdjGeo<TB>::smem_bytes));
        attr[dev] = true;
    }
    const int items = tab.item_prefix[tab.npairs];
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((items + kBackwardWarps - 1) / kBackwardWarps));
    cfg.blockDim = dim3(kBackwardWarps * 32);
    cfg.dynamicSmemBytes = AdjGeo<TB>::smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute a[1];
    a[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    a[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = a;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, fn, tab));
    return HS_OK;
}

static hs_status launch_adj_any(int TB, const AdjTable &tab, cudaStream_t s) {
    switch (TB) {
        case 1: return launch_adj<1>(tab, s);
        case 2: return launch_adj<2>(tab, s);
        case 3: return launch_adj<3>(tab, s);
        case 4: return launch_adj<4>(tab, s);
        case 5: return launch_adj<5>(tab, s);
    }
    HS_FAIL(HS_ERR_INVALID_ARG, "adjoint depth %d outside 1..%d", TB, kMaxTB);
}

// ------------------------------------------------------------------ per-pair finishing

struct FinishTable {
    const float *dIx[kMaxTrainPairs], *dIy[kMaxTrainPairs], *dIt[kMaxTrainPairs];
    float *dI0[kMaxTrainPairs], *dI1[kMaxTrainPairs];
    const float *alpha[kMaxTrainPairs];
    float *dalpha[kMaxTrainPairs];
    const double *a2part[kMaxTrainPairs];  // per pair: nslots partials
    int H[kMaxTrainPairs], W[kMaxTrainPairs], ld[kMaxTrainPairs];
    int npairs;
};

__device__ __forceinline__ int tap_src(int p, int o, int n, int xs[2]) {
    int c = 0;
    const int x = p - o;
    if (x >= 0 && x <= n - 1) xs[c++] = x;
    if (o == 1 && p == n - 1 && x != n - 1) xs[c++] = n - 1;  // (n-1) + 1 clamps to n-1
    return c;
}

// dI0 = Dx^T dIx + Dy^T dIy - Dt^T dIt; dI1 = ... + Dt^T dIt (taps (0,0) (1,0) (0,1) (1,1)).
__global__ void __launch_bounds__(256) batch_derivs_adjoint_kernel(const __grid_constant__ FinishTable ft) {
    const int i = blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= ft.npairs || x >= ft.W[i] || y >= ft.H[i]) return;
    const int H = ft.H[i], W = ft.W[i], ld = ft.ld[i];
    const float wx[4] = {-0.25f, 0.25f, -0.25f, 0.25f};
    const float wy[4] = {-0.25f, -0.25f, 0.25f, 0.25f};
    const int ox[4] = {0, 1, 0, 1}, oy[4] = {0, 0, 1, 1};
    float sc = 0.f, st = 0.f;
    for (int d = 0; d < 4; ++d) {
        int xs[2], ys[2];
        const int nx = tap_src(x, ox[d], W, xs), ny = tap_src(y, oy[d], H, ys);
        for (int jy = 0; jy < ny; ++jy)
            for (int jx = 0; jx < nx; ++jx) {
                const size_t q = (size_t)ys[jy] * ld + xs[jx];
                sc = fmaf(wx[d], __ldg(ft.dIx[i] + q), fmaf(wy[d], __ldg(ft.dIy[i] + q), sc));
                st = fmaf(0.25f, __ldg(ft.dIt[i] + q), st);
            }
    }
    const size_t o = (size_t)y * ld + x;
    ft.dI0[i][o] = sc - st;
    ft.dI1[i][o] = sc + st;
}

__global__ void __launch_bounds__(256) batch_fold_kernel(const __grid_constant__ FinishTable ft, int nparts) {
    __shared__ double sh[256];
    const int i = blockIdx.x;
    double s = 0.0;
    for (int e = threadIdx.x; e < nparts; e += blockDim.x) s += ft.a2part[i][e];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *ft.dalpha[i] = (float)(2.0 * (double)__ldg(ft.alpha[i]) * sh[0]);
}

// ------------------------------------------------------------------ host plan

// Where one pair's training buffers live: planes of pb bytes each.
//   derivs  Ix, Iy, It
//   ckpt    checkpoint c = x_{c k} (c = 0 .. nb; checkpoint nb is the final state) as (u, v)
//   states  two buffers (by interval parity) of x_{k_lo + j}, j = 1 .. k-1, as (u, v)
//   lam     two (lambda_u, lambda_v) buffers
//   acc     dIx, dIy, dIt accumulators
//   scratch two (u, v) buffers of the forward's inner passes
//   a2part  nslots doubles of dL/dalpha^2 partials
struct PairBufs {
    char *derivs, *ckpt, *states, *lam, *acc, *scratch;
    double *a2part;
    size_t pb;
    float *at(char *base, size_t i) const { return reinterpret_cast<float *>(base + i * pb); }
    float *deriv(int q) const { return at(derivs, q); }
    float *ck(int c, int comp) const { return at(ckpt, 2 * (size_t)c + comp); }
    int nstate;  // states per buffer (ckpt_every - 1)
    float *state(int j, int comp, int buf) const {
        return at(states, 2 * ((size_t)buf * nstate + (size_t)(j - 1)) + comp);
    }
    float *lamb(int buf, int comp) const { return at(lam, 2 * (size_t)buf + comp); }
    float *accum(int q) const { return at(acc, q); }
    float *scr(int buf, int comp) const { return at(scratch, 2 * (size_t)buf + comp); }
};

// adjoint work items of one pair in one launch, at most: all rows / rows per item (one wave
// of warps over the batch) + one partial segment per strip
static int adj_slots(int maxW) { return sm_count() * kAdjItemsPerSmMax + (maxW + kMinStripCols - 1) / kMinStripCols; }

struct TrainLayout {
    size_t pb;            // plane stride (bytes)
    size_t per_pair;      // bytes per pair
    int nb;               // checkpoint intervals
    // plane indices inside a pair's block
    size_t derivs, ckpt, states, lam, acc, scratch;
    size_t partials_off;  // after all pairs: [n][nslots] doubles
    int nslots;           // adjoint work items per pair and launch, upper bound
    size_t total;
};

static hs_status check_train_args(const hs_train_pair *pairs, int n, int iters, int ckpt_every,
                                  size_t *pbmax) {
    if (!pairs) HS_FAIL(HS_ERR_INVALID_ARG, "pairs is NULL");
    if (n < 1 || n > kMaxTrainPairs) HS_FAIL(HS_ERR_INVALID_ARG, "n=%d outside 1..%d", n, kMaxTrainPairs);
    if (iters < 1 || ckpt_every < 1)
        HS_FAIL(HS_ERR_INVALID_ARG, "iters=%d ckpt_every=%d must be >= 1", iters, ckpt_every);
    *pbmax = 0;
    for (int i = 0; i < n; ++i) {
        hs_status st = check_plane_geometry(pairs[i].H, pairs[i].W, pairs[i].ld);
        if (st != HS_OK) return st;
        if (pairs[i].reserved != 0) HS_FAIL(HS_ERR_INVALID_ARG, "pair %d: reserved must be zero", i);
        *pbmax = std::max(*pbmax, round_up(plane_bytes(pairs[i].H, pairs[i].ld), 256));
    }
    return HS_OK;
}

static hs_status train_layout(const hs_train_pair *pairs, int n, int iters, int ckpt_every,
                              TrainLayout &L) {
    hs_status st = check_train_args(pairs, n, iters, ckpt_every, &L.pb);
    if (st != HS_OK) return st;
    L.nb = (iters + ckpt_every - 1) / ckpt_every;
    L.derivs = 0;                                    // 3 planes
    L.ckpt = 3;                                      // (nb + 1) x 2 planes
    L.states = L.ckpt + 2 * (size_t)(L.nb + 1);      // 2 x (ckpt_every - 1) x 2 planes
    L.lam = L.states + 4 * (size_t)(ckpt_every - 1); // 2 x 2 planes
    L.acc = L.lam + 4;                               // 3 planes (dIx, dIy, dIt)
    L.scratch = L.acc + 3;                           // 2 x 2 planes
    L.per_pair = (L.scratch + 4) * L.pb;
    L.partials_off = (size_t)n * L.per_pair;
    int maxW = 1;
    for (int i = 0; i < n; ++i) maxW = std::max(maxW, pairs[i].W);
    L.nslots = adj_slots(maxW);
    L.total = L.partials_off + round_up((size_t)n * L.nslots * sizeof(double), 256);
    return HS_OK;
}

static PairBufs bufs_in_workspace(char *ws, const TrainLayout &L, int i) {
    char *b = ws + (size_t)i * L.per_pair;
    PairBufs B;
    B.pb = L.pb;
    B.derivs = b + L.derivs * L.pb;
    B.ckpt = b + L.ckpt * L.pb;
    B.states = b + L.states * L.pb;
    B.lam = b + L.lam * L.pb;
    B.acc = b + L.acc * L.pb;
    B.scratch = b + L.scratch * L.pb;
    B.a2part = reinterpret_cast<double *>(ws + L.partials_off) + (size_t)i * L.nslots;
    B.nstate = (int)((L.lam - L.states) / 4);
    return B;
}

static SweepParams base_params(const hs_train_pair &d, const PairBufs &B, const ResolvedConfig &rc,
                               int T) {
    SweepParams p;
    memset(&p, 0, sizeof(p));
    p.Ix = B.deriv(0);
    p.Iy = B.deriv(1);
    p.It = B.deriv(2);
    p.H = d.H;
    p.W = d.W;
    p.ld = d.ld;
    p.alpha2 = 0.f;
    p.alpha_dev = d.alpha;
    p.we = rc.we;
    p.wc = rc.wc;
    const int sc = strip_cols_for(T);
    p.nstrips = (d.W + sc - 1) / sc;
    p.dump = 0;
    return p;
}

// The training passes' layout is chosen like the per-pass sweep's, on the pixels of an image
// (the batch's average): the wide strips pay where images are large (measured: the 8 x 2048^2
// coarse-to-fine 1 % faster; 16 x 512^2 6 % slower, where 128-column strips cut 512 columns
// less evenly than 64-column ones).
static long pair_pixels(const hs_train_pair *pairs, int n) {
    long px = 0;
    for (int i = 0; i < n; ++i) px += (long)pairs[i].H * pairs[i].W;
    return px / std::max(n, 1);
}

// rows per work item for a table launch: about one wave of warps over all pairs.  In the
// 4-columns-per-lane layout the strips are re-cut and the wave holds the warps the wide
// kernel keeps resident (12 per SM to depth 4, 8 beyond).
static void set_segments(PassTable &tab, int T) {
    if (tab.wide)
        for (int i = 0; i < tab.npairs; ++i)
            tab.pair[i].nstrips = (tab.pair[i].W + strip_cols_wide(T) - 1) / strip_cols_wide(T);
    long rows = 0;
    for (int i = 0; i < tab.npairs; ++i) rows += (long)tab.pair[i].nstrips * tab.pair[i].H;
    const long target = (long)sm_count() * (tab.wide ? (T <= 4 ? 12 : 8) : 16);
    int L = (int)std::max(1L, (rows + target - 1) / target);
    L = std::max(L, 2 * T);
    tab.item_prefix[0] = 0;
    for (int i = 0; i < tab.npairs; ++i) {
        SweepParams &p = tab.pair[i];
        p.seg_rows = std::min(std::max(L, 8), p.H);
        p.nitems = p.nstrips * ((p.H + p.seg_rows - 1) / p.seg_rows);
        tab.item_prefix[i + 1] = tab.item_prefix[i] + p.nitems;
    }
}

// Forward with checkpoints: derivatives, x_0 = 0, then interval by interval; an interval's
// first pass reads checkpoint b and its last pass writes checkpoint b + 1.  The final state
// (checkpoint nb) is copied to the pairs' u, v.
static hs_status train_forward(const hs_train_pair *pairs, const PairBufs *bufs, int n, int iters,
                               int ckpt_every, const ResolvedConfig &rc, cudaStream_t s) {
    hs_status st;
    for (int i = 0; i < n; ++i) {
        const hs_train_pair &d = pairs[i];
        const PairBufs &B = bufs[i];
        if ((st = hs_derivs(d.I0, d.I1, d.H, d.W, d.ld, B.deriv(0), B.deriv(1), B.deriv(2), s)) != HS_OK)
            return st;
        HS_CUDA_CHECK(cudaMemsetAsync(B.ck(0, 0), 0, 2 * B.pb, s));  // x_0 = 0
    }
    const int T = rc.T;
    const bool wide = use_wide(rc, pair_pixels(pairs, n));
    const int nb = (iters + ckpt_every - 1) / ckpt_every;
    for (int b = 0; b < nb; ++b) {
        const int nsw = std::min(ckpt_every, iters - b * ckpt_every);
        const int passes = (nsw + T - 1) / T;
        for (int q = 0, done = 0; q < passes; ++q) {
            const int t = std::min(T, nsw - done);
            PassTable tab;
            memset(&tab, 0, sizeof(tab));
            tab.npairs = n;
            tab.wide = wide;
            for (int i = 0; i < n; ++i) {
                const PairBufs &B = bufs[i];
                SweepParams p = base_params(pairs[i], B, rc, t);
                p.u_in = q == 0 ? B.ck(b, 0) : B.scr((q - 1) & 1, 0);
                p.v_in = q == 0 ? B.ck(b, 1) : B.scr((q - 1) & 1, 1);
                p.u_out = q == passes - 1 ? B.ck(b + 1, 0) : B.scr(q & 1, 0);
                p.v_out = q == passes - 1 ? B.ck(b + 1, 1) : B.scr(q & 1, 1);
                tab.pair[i] = p;
            }
            set_segments(tab, t);
            if ((st = launch_table_any(t, rc.fast, tab, s)) != HS_OK) return st;
            done += t;
        }
    }
    for (int i = 0; i < n; ++i) {
        const size_t pl = plane_bytes(pairs[i].H, pairs[i].ld);
        HS_CUDA_CHECK(cudaMemcpyAsync(pairs[i].u, bufs[i].ck(nb, 0), pl, cudaMemcpyDeviceToDevice, s));
        HS_CUDA_CHECK(cudaMemcpyAsync(pairs[i].v, bufs[i].ck(nb, 1), pl, cudaMemcpyDeviceToDevice, s));
    }
    return HS_OK;
}

// A per-device side stream and events for the backward's two-stream schedule (created on
// first use outside any stream capture; kept until the process exits).  The mutex is held
// while a backward enqueues its work, so that calls from several host threads never
// interleave their records and waits on the shared events.
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t dump_done[2] = {}, adj_done[2] = {}, start = nullptr;
};
static std::mutex g_side_mu;
static SideStream g_side[64];

static hs_status side_stream(int dev, SideStream **out) {
    SideStream &S = g_side[dev];
    if (!S.s) {
        HS_CUDA_CHECK(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            HS_CUDA_CHECK(cudaEventCreateWithFlags(&S.dump_done[i], cudaEventDisableTiming));
            HS_CUDA_CHECK(cudaEventCreateWithFlags(&S.adj_done[i], cudaEventDisableTiming));
        }
        HS_CUDA_CHECK(cudaEventCreateWithFlags(&S.start, cudaEventDisableTiming));
    }
    *out = &S;
    return HS_OK;
}

// Backward of train_forward (the same buffers): per checkpoint interval in reverse, dump
// passes recompute the interval's states, then adjoint passes of balanced depth reverse its
// sweeps; last the transposed derivative stencils and the dalpha fold.
//
// The recompute of interval b-1 needs only its checkpoint, so it runs on a side stream while
// the adjoint passes of interval b run on the caller's stream: the two kernels' waves fill
// each other's tails.  The states are double-buffered by interval parity; the recompute of
// interval b-1 waits for the adjoint of interval b+1 (the last reader of its buffer), the
// adjoint of interval b waits for its recompute.  Without a side stream (first use inside a
// stream capture, or more than 64 devices) the same work runs in order on one stream.
static hs_status train_backward(const hs_train_pair *pairs, const PairBufs *bufs, int n, int iters,
                                int ckpt_every, int nslots, const ResolvedConfig &rc,
                                cudaStream_t s) {
    hs_status st;
    for (int i = 0; i < n; ++i) {
        const PairBufs &B = bufs[i];
        const size_t pl = plane_bytes(pairs[i].H, pairs[i].ld);
        HS_CUDA_CHECK(cudaMemcpyAsync(B.lamb(0, 0), pairs[i].dLdu, pl, cudaMemcpyDeviceToDevice, s));
        HS_CUDA_CHECK(cudaMemcpyAsync(B.lamb(0, 1), pairs[i].dLdv, pl, cudaMemcpyDeviceToDevice, s));
        HS_CUDA_CHECK(cudaMemsetAsync(B.accum(0), 0, 3 * B.pb, s));
        HS_CUDA_CHECK(cudaMemsetAsync(B.a2part, 0, (size_t)nslots * sizeof(double), s));
    }
    int cur = 0;  // lambda buffer holding dL/dx of the current sweep boundary
    const bool wide = use_wide(rc, pair_pixels(pairs, n));  // the dump passes' layout
    // adjoint depth: at most 4 (a 5-deep adjoint pass is register-bound and slower)
    const int TB = std::min(kAdjMaxDepth, std::max(1, rc.T));
    const int nb = (iters + ckpt_every - 1) / ckpt_every;

    // 1. states x_{k_lo+1} .. x_{k_lo+nsw-1} of interval b into state buffer b & 1
    auto dump = [&](int b, cudaStream_t ds) -> hs_status {
        const int nsw = std::min(ckpt_every, iters - b * ckpt_every);
        const int sb = b & 1;
        for (int done = 0; done < nsw - 1;) {
            const int t = std::min(kMaxDumpDepth, nsw - 1 - done);  // dump depth: 9 states = 5 + 4
            PassTable tab;
            memset(&tab, 0, sizeof(tab));
            tab.npairs = n;
            tab.wide = wide;
            for (int i = 0; i < n; ++i) {
                const PairBufs &B = bufs[i];
                SweepParams p = base_params(pairs[i], B, rc, t);
                p.u_in = done == 0 ? B.ck(b, 0) : B.state(done, 0, sb);
                p.v_in = done == 0 ? B.ck(b, 1) : B.state(done, 1, sb);
                p.dump = 1;
                for (int q = 0; q < t; ++q) {
                    p.dump_u[q] = B.state(done + q + 1, 0, sb);
                    p.dump_v[q] = B.state(done + q + 1, 1, sb);
                }
                p.u_out = p.dump_u[t - 1];
                p.v_out = p.dump_v[t - 1];
                tab.pair[i] = p;
            }
            set_segments(tab, t);
            hs_status e = launch_table_any(t, rc.fast, tab, ds);
            if (e != HS_OK) return e;
            done += t;
        }
        return HS_OK;
    };
    // 2. the adjoint sweeps m = iters .. 1 in ceil(iters / TB) passes of balanced depth
    //    (200 = 50 x 4).  A pass may span two checkpoint intervals: x_m is checkpoint
    //    m / k when k divides m (or m = iters), else state m - b k of interval b = (m-1)/k.
    auto interval_of = [&](int m) { return (m - 1) / ckpt_every; };
    auto nsw_of = [&](int b) { return std::min(ckpt_every, iters - b * ckpt_every); };
    auto state_ptr = [&](const PairBufs &B, int m, int comp) -> const float * {
        const int b = interval_of(m), j = m - b * ckpt_every;
        return j == nsw_of(b) ? B.ck(b + 1, comp) : B.state(j, comp, b & 1);
    };
    auto adjoint_pass = [&](int jhi, int tb, cudaStream_t as) -> hs_status {
        AdjTable tab;
        memset(&tab, 0, sizeof(tab));
        tab.npairs = n;
        tab.we = rc.we;
        tab.wc = rc.wc;
        long rows = 0;
        for (int i = 0; i < n; ++i) rows += (long)((pairs[i].W + strip_cols_for(tb) - 1) / strip_cols_for(tb)) * pairs[i].H;
        const long target = (long)sm_count() * adj_res_warps(tb);
        int Lr = (int)std::max(1L, (rows + target - 1) / target);
        Lr = std::max(Lr, std::max(8, 2 * tb));
        tab.item_prefix[0] = 0;
        for (int i = 0; i < n; ++i) {
            const hs_train_pair &d = pairs[i];
            const PairBufs &B = bufs[i];
            AdjPair &P = tab.pair[i];
            P.Ix = B.deriv(0);
            P.Iy = B.deriv(1);
            P.It = B.deriv(2);
            P.lu_in = B.lamb(cur, 0);
            P.lv_in = B.lamb(cur, 1);
            P.lu_out = B.lamb(cur ^ 1, 0);
            P.lv_out = B.lamb(cur ^ 1, 1);
            for (int qq = 0; qq < tb; ++qq) {  // stage qq reverses sweep jhi - qq
                P.xu[qq] = state_ptr(B, jhi - qq, 0);
                P.xv[qq] = state_ptr(B, jhi - qq, 1);
            }
            P.aIx = B.accum(0);
            P.aIy = B.accum(1);
            P.aIt = B.accum(2);
            P.a2part = B.a2part;
            P.alpha_dev = d.alpha;
            P.H = d.H;
            P.W = d.W;
            P.ld = d.ld;
            P.nstrips = (d.W + strip_cols_for(tb) - 1) / strip_cols_for(tb);
            P.seg_rows = std::min(Lr, d.H);
            const int items = P.nstrips * ((d.H + P.seg_rows - 1) / P.seg_rows);
            if (items > nslots) HS_FAIL(HS_ERR_INVALID_ARG, "adjoint items %d > slots %d", items, nslots);
            tab.item_prefix[i + 1] = tab.item_prefix[i] + items;
        }
        hs_status e = launch_adj_any(tb, tab, as);
        if (e != HS_OK) return e;
        cur ^= 1;
        return HS_OK;
    };

    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    HS_CUDA_CHECK(cudaStreamIsCapturing(s, &cap));
    std::unique_lock<std::mutex> lock(g_side_mu);
    SideStream *S = nullptr;
    if (nb > 1 && dev < 64 && (g_side[dev].s || cap == cudaStreamCaptureStatusNone)) {
        if ((st = side_stream(dev, &S)) != HS_OK) return st;
    } else {
        lock.unlock();
    }
    // Schedule.  Interval b's states are recomputed (dump) before the first pass that reads
    // them; its buffer (parity b & 1) is free again once the last pass reading interval
    // b+2 has run.  With the side stream the recompute runs up to two intervals ahead of the
    // passes: dump(b) waits for the passes of b+2 to finish (event adj_done[b & 1]) and the
    // passes reading b wait for dump(b) (event dump_done[b & 1]).
    const cudaStream_t ds = S ? S->s : s;
    int next_dump = nb - 1;  // intervals >= next_dump have their dump issued
    auto issue_dump = [&](int b) -> hs_status {
        if (S && b + 2 <= nb - 1) HS_CUDA_CHECK(cudaStreamWaitEvent(ds, S->adj_done[b & 1], 0));
        hs_status e = dump(b, ds);
        if (e != HS_OK) return e;
        if (S) HS_CUDA_CHECK(cudaEventRecord(S->dump_done[b & 1], ds));
        next_dump = b - 1;
        return HS_OK;
    };
    if (S) {
        // the side stream starts after everything the caller queued before this call
        HS_CUDA_CHECK(cudaEventRecord(S->start, s));
        HS_CUDA_CHECK(cudaStreamWaitEvent(ds, S->start, 0));
        if ((st = issue_dump(nb - 1)) != HS_OK) return st;
        if (nb >= 2 && (st = issue_dump(nb - 2)) != HS_OK) return st;
    }
    const int npass = (iters + TB - 1) / TB;
    for (int jhi = iters, q = 0; jhi > 0; ++q) {
        const int tb = (jhi + (npass - q) - 1) / (npass - q);
        const int jlo = jhi - tb + 1;
        const int b_hi = interval_of(jhi), b_lo = interval_of(jlo);
        // the recompute of every interval whose states this pass reads (at most two adjacent
        // intervals for depth <= 4 and k >= 2; none for k = 1); in order without a side stream
        for (int b = b_hi; b >= b_lo; --b) {
            bool reads = false;
            for (int m = jlo; m <= jhi; ++m)
                reads |= interval_of(m) == b && m - b * ckpt_every != nsw_of(b);
            if (!reads) continue;
            if (!S) {
                while (next_dump >= b)
                    if ((st = issue_dump(next_dump)) != HS_OK) return st;
            } else {
                if (next_dump >= b) HS_FAIL(HS_ERR_INVALID_ARG, "internal: interval %d read before its recompute", b);
                HS_CUDA_CHECK(cudaStreamWaitEvent(s, S->dump_done[b & 1], 0));
            }
        }
        if ((st = adjoint_pass(jhi, tb, s)) != HS_OK) return st;
        // intervals no later pass reads: above b_lo, and b_lo itself once its first sweep is
        // reversed; their buffers go to the recompute two intervals further down
        const int b_done_lo = (jlo == b_lo * ckpt_every + 1) ? b_lo : b_lo + 1;
        for (int b = b_hi; b >= b_done_lo; --b) {
            if (!S) continue;
            HS_CUDA_CHECK(cudaEventRecord(S->adj_done[b & 1], s));
            if (b - 2 >= 0 && next_dump == b - 2 && (st = issue_dump(b - 2)) != HS_OK) return st;
        }
        jhi -= tb;
    }

    // 3. transposed derivative stencils and dalpha
    FinishTable ft;
    memset(&ft, 0, sizeof(ft));
    ft.npairs = n;
    int maxW = 1, maxH = 1;
    for (int i = 0; i < n; ++i) {
        const PairBufs &B = bufs[i];
        ft.dIx[i] = B.accum(0);
        ft.dIy[i] = B.accum(1);
        ft.dIt[i] = B.accum(2);
        ft.a2part[i] = B.a2part;
        ft.dI0[i] = pairs[i].dI0;
        ft.dI1[i] = pairs[i].dI1;
        ft.alpha[i] = pairs[i].alpha;
        ft.dalpha[i] = pairs[i].dalpha;
        ft.H[i] = pairs[i].H;
        ft.W[i] = pairs[i].W;
        ft.ld[i] = pairs[i].ld;
        maxW = std::max(maxW, pairs[i].W);
        maxH = std::max(maxH, pairs[i].H);
    }
    batch_derivs_adjoint_kernel<<<dim3((maxW + 63) / 64, (maxH + 3) / 4, n), dim3(64, 4), 0, s>>>(ft);
    HS_LAUNCH_CHECK("batch_derivs_adjoint_kernel");
    batch_fold_kernel<<<n, 256, 0, s>>>(ft, nslots);
    HS_LAUNCH_CHECK("batch_fold_kernel");
    return HS_OK;
}

static size_t plane_stride(int H, int ld) { return round_up(plane_bytes(H, ld), 256); }

}  // namespace hs

using namespace hs;

extern "C" {

size_t hs_train_workspace_bytes(const hs_train_pair *pairs, int n, int iters, int ckpt_every) {
    TrainLayout L;
    if (train_layout(pairs, n, iters, ckpt_every, L) != HS_OK) return 0;
    return L.total;
}

hs_status hs_forward_train_batched(const hs_train_pair *pairs, int n, int iters, int ckpt_every,
                                   void *workspace, size_t workspace_bytes, const hs_config *cfg,
                                   void *stream) {
    clear_error();
    TrainLayout L;
    hs_status st = train_layout(pairs, n, iters, ckpt_every, L);
    if (st != HS_OK) return st;
    ResolvedConfig rc;
    if ((st = resolve_config(cfg, &rc)) != HS_OK) return st;
    if (!workspace || workspace_bytes < L.total)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, L.total);
    if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
        HS_FAIL(HS_ERR_ALIGNMENT, "workspace is not 256-byte aligned");
    for (int i = 0; i < n; ++i) {
        const void *pl[4] = {pairs[i].I0, pairs[i].I1, pairs[i].u, pairs[i].v};
        const char *nm[4] = {"I0", "I1", "u", "v"};
        for (int q = 0; q < 4; ++q)
            if ((st = check_plane(pl[q], nm[q])) != HS_OK) return st;
        if (!pairs[i].alpha) HS_FAIL(HS_ERR_INVALID_ARG, "pair %d: alpha (device) is NULL", i);
    }
    std::vector<PairBufs> bufs(n);
    for (int i = 0; i < n; ++i) bufs[i] = bufs_in_workspace(reinterpret_cast<char *>(workspace), L, i);
    return train_forward(pairs, bufs.data(), n, iters, ckpt_every, rc, (cudaStream_t)stream);
}

hs_status hs_backward_batched(const hs_train_pair *pairs, int n, int iters, int ckpt_every,
                              void *workspace, size_t workspace_bytes, const hs_config *cfg,
                              void *stream) {
    clear_error();
    TrainLayout L;
    hs_status st = train_layout(pairs, n, iters, ckpt_every, L);
    if (st != HS_OK) return st;
    ResolvedConfig rc;
    if ((st = resolve_config(cfg, &rc)) != HS_OK) return st;
    if (!workspace || workspace_bytes < L.total)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, L.total);
    for (int i = 0; i < n; ++i) {
        const void *pl[4] = {pairs[i].dLdu, pairs[i].dLdv, pairs[i].dI0, pairs[i].dI1};
        const char *nm[4] = {"dLdu", "dLdv", "dI0", "dI1"};
        for (int q = 0; q < 4; ++q)
            if ((st = check_plane(pl[q], nm[q])) != HS_OK) return st;
        if (!pairs[i].alpha || !pairs[i].dalpha)
            HS_FAIL(HS_ERR_INVALID_ARG, "pair %d: alpha / dalpha (device) NULL", i);
    }
    std::vector<PairBufs> bufs(n);
    for (int i = 0; i < n; ++i) bufs[i] = bufs_in_workspace(reinterpret_cast<char *>(workspace), L, i);
    return train_backward(pairs, bufs.data(), n, iters, ckpt_every, L.nslots, rc, (cudaStream_t)stream);
}

// ---- the single-pair form: the same passes on caller-held derivative and checkpoint
// buffers (n = 1)

size_t hs_derivs_bytes(int H, int W, int ld) {
    (void)W;
    if (H < 1 || ld < 1) return 0;
    return 3 * plane_stride(H, ld);
}

size_t hs_checkpoint_bytes(int H, int W, int ld, int iters, int ckpt_every) {
    (void)W;
    if (H < 1 || ld < 1 || iters < 0 || ckpt_every < 1) return 0;
    if (iters == 0) return 0;
    const size_t nb = (size_t)((iters + ckpt_every - 1) / ckpt_every);
    return (nb + 1) * 2 * plane_stride(H, ld);
}

size_t hs_forward_train_workspace_bytes(int H, int W, int ld) {
    (void)W;
    if (H < 1 || ld < 1) return 0;
    return 4 * plane_stride(H, ld);
}

size_t hs_backward_workspace_bytes(int H, int W, int ld, int ckpt_every) {
    if (H < 1 || W < 1 || ld < 1 || ckpt_every < 1) return 0;
    // states 2 x (ckpt_every - 1) x 2, lambda 2 x 2, accumulators 3 planes, then the partials
    const size_t planes = 4 * (size_t)(ckpt_every - 1) + 4 + 3;
    return planes * plane_stride(H, ld) + round_up((size_t)adj_slots(W) * sizeof(double), 256);
}

hs_status hs_forward_train(const float *I0, const float *I1, int H, int W, int ld,
                           const float *alpha, int iters, int ckpt_every, float *u, float *v,
                           float *derivs, float *ckpt, void *workspace, size_t workspace_bytes,
                           const hs_config *cfg, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *planes[5] = {I0, I1, u, v, derivs};
    const char *names[5] = {"I0", "I1", "u", "v", "derivs"};
    for (int i = 0; i < 5; ++i)
        if ((st = check_plane(planes[i], names[i])) != HS_OK) return st;
    if (!alpha) HS_FAIL(HS_ERR_INVALID_ARG, "alpha (device pointer) is NULL");
    if (iters < 0 || ckpt_every < 1) HS_FAIL(HS_ERR_INVALID_ARG, "iters=%d ckpt_every=%d", iters, ckpt_every);
    ResolvedConfig rc;
    if ((st = resolve_config(cfg, &rc)) != HS_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t pb = plane_stride(H, ld);
    if (iters == 0) {  // nothing to checkpoint: the derivatives and u = v = 0
        char *dv = reinterpret_cast<char *>(derivs);
        if ((st = hs_derivs(I0, I1, H, W, ld, reinterpret_cast<float *>(dv),
                            reinterpret_cast<float *>(dv + pb), reinterpret_cast<float *>(dv + 2 * pb),
                            stream)) != HS_OK)
            return st;
        HS_CUDA_CHECK(cudaMemsetAsync(u, 0, plane_bytes(H, ld), s));
        HS_CUDA_CHECK(cudaMemsetAsync(v, 0, plane_bytes(H, ld), s));
        return HS_OK;
    }
    if ((st = check_plane(ckpt, "ckpt")) != HS_OK) return st;
    const size_t need = hs_forward_train_workspace_bytes(H, W, ld);
    if (!workspace || workspace_bytes < need)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, need);
    if (!aligned16(workspace)) HS_FAIL(HS_ERR_ALIGNMENT, "workspace is not 16-byte aligned");
    hs_train_pair d;
    memset(&d, 0, sizeof(d));
    d.I0 = I0;
    d.I1 = I1;
    d.u = u;
    d.v = v;
    d.alpha = alpha;
    d.H = H;
    d.W = W;
    d.ld = ld;
    PairBufs B;
    memset(&B, 0, sizeof(B));
    B.pb = pb;
    B.derivs = reinterpret_cast<char *>(derivs);
    B.ckpt = reinterpret_cast<char *>(ckpt);
    B.scratch = reinterpret_cast<char *>(workspace);
    return train_forward(&d, &B, 1, iters, ckpt_every, rc, s);
}

hs_status hs_backward(const float *derivs, int H, int W, int ld, const float *alpha, int iters,
                      int ckpt_every, const float *ckpt, const float *dLdu, const float *dLdv,
                      float *dI0, float *dI1, float *dalpha, void *workspace,
                      size_t workspace_bytes, const hs_config *cfg, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const void *planes[6] = {derivs, dLdu, dLdv, dI0, dI1, workspace};
    const char *names[6] = {"derivs", "dLdu", "dLdv", "dI0", "dI1", "workspace"};
    for (int i = 0; i < 6; ++i)
        if ((st = check_plane(planes[i], names[i])) != HS_OK) return st;
    if (!alpha || !dalpha) HS_FAIL(HS_ERR_INVALID_ARG, "alpha / dalpha (device pointers) NULL");
    if (iters < 0 || ckpt_every < 1) HS_FAIL(HS_ERR_INVALID_ARG, "iters=%d ckpt_every=%d", iters, ckpt_every);
    if (iters > 0 && (st = check_plane(ckpt, "ckpt")) != HS_OK) return st;
    ResolvedConfig rc;
    if ((st = resolve_config(cfg, &rc)) != HS_OK) return st;
    const size_t need = hs_backward_workspace_bytes(H, W, ld, ckpt_every);
    if (workspace_bytes < need)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, need);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t pb = plane_stride(H, ld);
    hs_train_pair d;
    memset(&d, 0, sizeof(d));
    d.alpha = alpha;
    d.dLdu = dLdu;
    d.dLdv = dLdv;
    d.dI0 = dI0;
    d.dI1 = dI1;
    d.dalpha = dalpha;
    d.H = H;
    d.W = W;
    d.ld = ld;
    if (iters == 0) {  // (u, v) = 0 whatever the images: no gradient reaches them
        HS_CUDA_CHECK(cudaMemsetAsync(dI0, 0, plane_bytes(H, ld), s));
        HS_CUDA_CHECK(cudaMemsetAsync(dI1, 0, plane_bytes(H, ld), s));
        HS_CUDA_CHECK(cudaMemsetAsync(dalpha, 0, sizeof(float), s));
        return HS_OK;
    }
    char *ws = reinterpret_cast<char *>(workspace);
    const size_t nst = 4 * (size_t)(ckpt_every - 1);
    PairBufs B;
    memset(&B, 0, sizeof(B));
    B.pb = pb;
    B.derivs = const_cast<char *>(reinterpret_cast<const char *>(derivs));
    B.ckpt = const_cast<char *>(reinterpret_cast<const char *>(ckpt));
    B.states = ws;
    B.lam = ws + nst * pb;
    B.acc = ws + (nst + 4) * pb;
    B.a2part = reinterpret_cast<double *>(ws + (nst + 7) * pb);
    B.nstate = ckpt_every - 1;
    return train_backward(&d, &B, 1, iters, ckpt_every, adj_slots(W), rc, s);
}

}  // extern "C"
