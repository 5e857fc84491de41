// hs_sweep.cu -- the per-pass launch of the temporally blocked Horn-Schunck sweep and
// the plain entry points hs_sweeps / hs_forward.  The streaming device code is in
// hs_stream.cuh.
#include <algorithm>

#include "hs_stream4.cuh"

namespace hs {

// Resident warps per SM the register budget is sized for (shared memory allows it too).
// (Measured: capping registers for more warps costs more ILP than it gains.)
constexpr int res_warps(int T) { return T <= 4 ? 16 : (T <= 6 ? 12 : 8); }

template <int T, bool FAST, bool UNR>
__global__ void __launch_bounds__(kPassWarps * 32, res_warps(T) / kPassWarps)
    hs_stream_kernel(const SweepParams p) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *wbase = reinterpret_cast<float *>(smem4) + warp * Geo<T>::warp_floats;

    griddep_launch_dependents();
    griddep_wait();

    const int item = blockIdx.x * kPassWarps + warp;
    if (item >= p.nitems) return;  // warp-uniform
    Item it;
    init_item<T>(it, p, item % p.nstrips, item / p.nstrips, lane, wbase);
    run_item<T, FAST, false, UNR>(p, it);
}

// The fast form in the wide layout (hs_stream4.cuh).
constexpr int res_warps_w(int T) { return T <= 4 ? 12 : 8; }

template <int T, bool UNR>
__global__ void __launch_bounds__(kPassWarps * 32, res_warps_w(T) / kPassWarps)
    hs_stream_w_kernel(const SweepParams p) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *wbase = reinterpret_cast<float *>(smem4) + warp * GeoW<T>::warp_floats;

    griddep_launch_dependents();
    griddep_wait();

    const int item = blockIdx.x * kPassWarps + warp;
    if (item >= p.nitems) return;  // warp-uniform
    ItemW it;
    init_item_w<T>(it, p, item % p.nstrips, item / p.nstrips, lane, wbase);
    run_item_w<T, false, UNR>(p, it);
}

// ------------------------------------------------------------------ host side

using KernelFn = void (*)(const SweepParams);

static hs_status launch_kernel(KernelFn fn, int smem, bool *attr_set, const SweepParams &pp,
                               cudaStream_t stream) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_set[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_set[dev] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((pp.nitems + kPassWarps - 1) / kPassWarps));
    cfg.blockDim = dim3(kPassWarps * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, fn, pp));
    return HS_OK;
}

// Images below this size (L2-resident) run the wide kernel's main loop rolled, larger ones
// unrolled two steps (stream_item_w); measured on B200 (fast form, T = 7): 1080p 521 against
// 502 Gpix-it/s rolled, 2048^2 605 against 608, 2560x1440 536 against 546, 4096^2 900 against
// 918.
constexpr long kUnrollPixels = 3000000;

template <int T>
static hs_status launch_one_w(const SweepParams &pp, cudaStream_t stream) {
    static bool attr_set[64] = {}, attr_set_r[64] = {};
    constexpr int smem = kPassWarps * GeoW<T>::warp_floats * (int)sizeof(float);
    if ((long)pp.H * pp.W >= kUnrollPixels)
        return launch_kernel(hs_stream_w_kernel<T, true>, smem, attr_set, pp, stream);
    return launch_kernel(hs_stream_w_kernel<T, false>, smem, attr_set_r, pp, stream);
}

int strip_cols_wide(int T) {
    switch (T) {
        case 1: return GeoW<1>::strip;
        case 2: return GeoW<2>::strip;
        case 3: return GeoW<3>::strip;
        case 4: return GeoW<4>::strip;
        case 5: return GeoW<5>::strip;
        case 6: return GeoW<6>::strip;
        case 7: return GeoW<7>::strip;
        default: return GeoW<8>::strip;
    }
}

static hs_status launch_pass_w(int T, const SweepParams &pp, cudaStream_t s) {
    switch (T) {
        case 1: return launch_one_w<1>(pp, s);
        case 2: return launch_one_w<2>(pp, s);
        case 3: return launch_one_w<3>(pp, s);
        case 4: return launch_one_w<4>(pp, s);
        case 5: return launch_one_w<5>(pp, s);
        case 6: return launch_one_w<6>(pp, s);
        case 7: return launch_one_w<7>(pp, s);
        case 8: return launch_one_w<8>(pp, s);
    }
    HS_FAIL(HS_ERR_INVALID_ARG, "sweeps_per_pass=%d outside 1..%d", T, HS_MAX_SWEEPS_PER_PASS);
}

template <int T, bool FAST>
static hs_status launch_one(const SweepParams &pp, cudaStream_t stream) {
    using G = Geo<T>;
    // rolled main loop from depth 3 at every image size (measured on B200, exact form: 1080p
    // T = 4 262 against 257 Gpix-it/s, T = 5 225 against 200; 2048^2 T = 6 278 against 237;
    // 3840x2160 T = 6 319 against 295; 4096^2 T = 4 390 against 386; fast form at 1080p T = 4
    // 391 against 359); at T = 2 the unrolled loop is faster (1080p exact: 251 against 211)
    auto fn = hs_stream_kernel<T, FAST, (T <= 2)>;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_set[dev]) {
        HS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kPassWarps * G::warp_floats * (int)sizeof(float)));
        attr_set[dev] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((pp.nitems + kPassWarps - 1) / kPassWarps));
    cfg.blockDim = dim3(kPassWarps * 32);
    cfg.dynamicSmemBytes = kPassWarps * G::warp_floats * (int)sizeof(float);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, fn, pp));
    return HS_OK;
}

int strip_cols_for(int T) {
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

hs_status launch_pass(int T, bool fast, const SweepParams &pp, cudaStream_t s) {
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
static int seg_rows_for(int H, int nstrips, int T, long warps_per_sm) {
    const long target = (long)sm_count() * warps_per_sm;
    long nseg = (target + nstrips - 1) / nstrips;
    if (nseg < 1) nseg = 1;
    int L = (int)((H + nseg - 1) / nseg);
    L = std::max(L, 2 * T);
    L = std::max(L, 8);
    return std::min(L, H);
}

int default_seg_rows(int H, int nstrips, int T) { return seg_rows_for(H, nstrips, T, 16); }

// Measured on B200: in a launch of several pairs (the batch and the training passes) the wide
// layout wins from about a 1080p image up (4096^2: 700 vs 592 Gpix-it/s), the narrow one below
// (more strips for the SMs on small images).  For one pair in one-warp CTAs the crossing lies
// near 250 kpx: at the default segments, as a fraction of the fastest tuned time, 480x640 runs
// 1.01 wide (T = 6) against 1.26 narrow, 512^2 1.05 against 1.12, 256^2 1.14 against 1.00.
constexpr long kWideAutoPixels = 2000000;
constexpr long kWideAutoPixelsPair = 250000;

static bool use_wide_at(const ResolvedConfig &rc, long pixels, long threshold) {
    if (!rc.fast) return false;
    if (rc.layout == 2) return true;
    if (rc.layout == 1) return false;
    return pixels >= threshold;
}
bool use_wide(const ResolvedConfig &rc, long pixels) { return use_wide_at(rc, pixels, kWideAutoPixels); }

hs_status resolve_config(const hs_config *cfg, ResolvedConfig *out) {
    hs_config c = {};
    if (cfg) c = *cfg;
    for (int i = 0; i < 2; ++i)
        if (c.reserved[i] != 0) HS_FAIL(HS_ERR_INVALID_ARG, "hs_config.reserved must be zero");
    if (c.layout < 0 || c.layout > 2) HS_FAIL(HS_ERR_INVALID_ARG, "hs_config.layout=%d outside 0..2", c.layout);
    if (c.layout == 2 && c.fast_math == 0)
        HS_FAIL(HS_ERR_INVALID_ARG, "hs_config.layout=2 needs fast_math (the exact form has 2 columns per lane)");
    out->layout = c.layout;
    out->fast = c.fast_math != 0;
    out->T = c.sweeps_per_pass > 0 ? c.sweeps_per_pass : 4;
    out->T_default = c.sweeps_per_pass == 0;
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


// The depth the per-pair sweep runs when hs_config.sweeps_per_pass is 0.  The table rounds
// the depths that are fastest on B200 at the default rows per segment and layout, by image
// size; at each of 240x320, 256^2, 480x640, 512^2, 1280x720, 1920x1080, 2048^2 and 4096^2 it
// runs within 6 % of the fastest tuned configuration (16 % at 512^2 in the fast form), fast
// and exact form.
void apply_shape_default(ResolvedConfig &rc, int H, int W) {
    if (!rc.T_default) return;
    const long px = (long)H * W;
    if (rc.fast)
        rc.T = px < 250000 ? 4 : px < 600000 ? 6 : px < 1500000 ? 5 : 7;
    else
        rc.T = px < 200000 ? 4 : px < 600000 ? 5 : 4;
}

// Runs `iters` sweeps.  State starts in (u0, v0) if `start_in_user`, else in (u1, v1);
// the final state always lands in (u0, v0).
hs_status run_passes_dev(const float *Ix, const float *Iy, const float *It, int H, int W, int ld,
                         float alpha2, const float *alpha_dev, int iters, float *u0, float *v0,
                         float *u1, float *v1, const ResolvedConfig &rc, cudaStream_t stream) {
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
        pp.alpha_dev = alpha_dev;
        pp.dump = 0;
        pp.we = rc.we; pp.wc = rc.wc;
        const bool wide = use_wide_at(rc, (long)H * W, kWideAutoPixelsPair);
        const int sc = wide ? strip_cols_wide(t) : strip_cols_for(t);
        pp.nstrips = (W + sc - 1) / sc;
        pp.seg_rows = rc.seg_rows > 0 ? std::min(rc.seg_rows, H)
                                      : seg_rows_for(H, pp.nstrips, t, wide ? res_warps_w(t) : 16);
        const int nseg = (H + pp.seg_rows - 1) / pp.seg_rows;
        pp.nitems = pp.nstrips * nseg;
        hs_status st = wide ? launch_pass_w(t, pp, stream) : launch_pass(t, rc.fast, pp, stream);
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
    apply_shape_default(rc, H, W);
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
    return run_passes_dev(Ix, Iy, It, H, W, ld, alpha2, nullptr, iters, u, v, u1, v1, rc, s);
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
    apply_shape_default(rc, H, W);
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
    return run_passes_dev(Ix, Iy, It, H, W, ld, alpha2, nullptr, iters, u, v, u1, v1, rc, s);
}

}  // extern "C"
