// hs_batch.cu -- many Horn-Schunck pairs of uneven size in one persistent launch.
//
// Work list.  Every (pass, pair, segment, strip) tile of every pair's full T-sweep passes
// is one work item; the tiles of one (pair, pass) unit are consecutive, segment-major.
// Units are ordered by the pair's progress, pass p of a pair with P passes at p / P
// (ties by pair): a pair of 20 passes contributes a pass wherever a pair of 100 passes has
// run 5, so the pairs with few passes are spread over the whole launch instead of all
// finishing early and leaving the longest chains to run alone at the end.  A one-block
// set-up kernel ranks the units (batch_order_kernel).  Warps take items from a global
// atomic counter; a warp runs its item with the streaming sweep of hs_stream.cuh and then
// publishes "tile done through pass p".
//
// Dependencies.  A tile's pass p reads rows and columns of pass p-1 reaching at most
// one tile beyond its own in each direction (the halo is at most T rows and columns, a
// segment is at least T rows and a strip at least 48 columns), and overwrites the buffer
// those pass p-1 tiles read.  So pass p of tile (g, s) waits until its 3x3 neighbour
// tiles have completed pass p-1.  A pair's pass p-1 unit comes before its pass p unit
// (p / P grows with p), so every tile an item waits on has a smaller item number; it was
// taken earlier by a running warp that waits only on smaller numbers still: the waits
// always end.  Each wait is nevertheless bounded; a wait that gives up records
// HS_ERR_TIMEOUT in the device status word and raises an abort flag on which every warp
// stops.  Completion is published with a release store after the tile's writes and the
// waits use acquire loads; rows are copied with cp.async.cg (L2), so no stale L1 line
// is read.
//
// A pair whose sweep count is not a multiple of T finishes with one more, shorter pass
// launched per pair after the persistent kernel.
#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "hs_stream4.cuh"

namespace hs {

constexpr int kMaxBatch = HS_MAX_BATCH;
constexpr int kHeaderBytes = 256;  // queue counters (2-column and 4-column launch), status, abort flag
constexpr unsigned long long kWaitPolls = 1ull << 22;  // bounded wait (seconds, at most)

struct BatchPair {
    const float *Ix, *Iy, *It;
    float *U[2], *V[2];  // [0] = caller's output, [1] = scratch
    unsigned *progress;  // per tile: passes completed
    int H, W, ld;
    float alpha2;
    int passes;  // full T-sweep passes in the persistent kernel
    int start;   // buffer the first pass reads
    int nstrips, seg_rows, items;
};

// Units (pair, pass) ranked by (p * kOrderScale / P, pair): kOrderScale exceeds every
// pass count, so the keys of one pair's passes are distinct and increasing.
constexpr long long kOrderScale = 1LL << 30;

struct BatchParams {
    BatchPair pair[kMaxBatch];
    int unit_prefix[kMaxBatch + 1];  // units of pairs before pair r (host order)
    int nunits;                      // all units = unit_prefix[npairs]
    int *unit_pp;                    // [nunits]: (pass << 8) | pair, in work order
    int *unit_first;                 // [nunits + 1]: first item of each unit, then the total
    int npairs, total_items;
    float we, wc;
    unsigned *queue;
    int *status;
    unsigned *abort_flag;
};

// Rank every unit of the launch and the first item of each (one block).  The rank of unit
// (r, p) with key K = floor(p S / P_r) is the number of units (j, q) with
// (floor(q S / P_j), j) < (K, r): for pair j the q with floor(q S / P_j) < K + [j < r], i.e.
// q < (K + [j < r]) P_j / S, so ceil((K + [j < r]) P_j / S) of them (at most P_j).
__global__ void __launch_bounds__(1024) batch_order_kernel(const __grid_constant__ BatchParams bp) {
    for (int u = threadIdx.x; u < bp.nunits; u += blockDim.x) {
        int r = 0;
        while (r + 1 < bp.npairs && bp.unit_prefix[r + 1] <= u) ++r;
        const int p = u - bp.unit_prefix[r];
        const long long K = (long long)p * kOrderScale / bp.pair[r].passes;
        long long rank = 0, first = 0;
        for (int j = 0; j < bp.npairs; ++j) {
            const long long Pj = bp.pair[j].passes;
            if (Pj == 0) continue;
            const long long a = (K + (j < r ? 1 : 0)) * Pj;
            const long long c = min(Pj, (a + kOrderScale - 1) / kOrderScale);
            rank += c;
            first += c * bp.pair[j].items;
        }
        bp.unit_pp[rank] = (p << 8) | r;
        bp.unit_first[rank] = (int)first;
    }
    if (threadIdx.x == 0) bp.unit_first[bp.nunits] = bp.total_items;
}

struct DerivParams {
    const float *I0[kMaxBatch], *I1[kMaxBatch];
    float *Ix[kMaxBatch], *Iy[kMaxBatch], *It[kMaxBatch];
    float *U0[kMaxBatch], *V0[kMaxBatch];  // initial-state buffers, zeroed here
    int H[kMaxBatch], W[kMaxBatch], ld[kMaxBatch];
    int npairs;
};

// Derivatives of every pair and u = v = 0 in the buffer each pair's first pass reads.
__global__ void __launch_bounds__(256) batch_derivs_kernel(const __grid_constant__ DerivParams dp) {
    const int i = blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= dp.npairs || x >= dp.W[i] || y >= dp.H[i]) return;
    const size_t o = (size_t)y * dp.ld[i] + x;
    hs_derivs_at(dp.I0[i], dp.I1[i], x, y, dp.H[i], dp.W[i], dp.ld[i], dp.Ix[i][o], dp.Iy[i][o],
                 dp.It[i][o]);
    dp.U0[i][o] = 0.0f;
    dp.V0[i][o] = 0.0f;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded warp-wide wait: each lane watches `flag` (nullptr: nothing to wait for) until it
// reaches `need`; one round of acquire loads checks every lane's flag, with an exponential
// nanosleep back-off (32 .. 256 ns) between rounds.  Gives up (false on every lane) after
// `max_polls` rounds or when *abort_flag is raised.
__device__ bool warp_wait_ge(const unsigned *flag, unsigned need, const unsigned *abort_flag,
                             unsigned long long max_polls, int lane) {
    unsigned long long polls = 0;
    unsigned ns = 32;
    for (;;) {
        const bool done = flag == nullptr || ld_acquire(flag) >= need;
        if (__all_sync(kFull, done)) return true;
        ++polls;
        int stop = 0;
        if (lane == 0)
            stop = polls > max_polls || ((polls & 63) == 0 && *(volatile const unsigned *)abort_flag);
        if (__shfl_sync(kFull, stop, 0)) return false;
        __nanosleep(ns);
        ns = min(ns * 2, 256u);
    }
}

// The warp waits until tiles (seg+-1, strip+-1) of pair P have completed `need` passes:
// lane i < 9 watches neighbour i.  Returns false if the wait gave up or another warp aborted.
__device__ bool wait_neighbours(const BatchPair &P, int seg, int strip, unsigned need,
                                const unsigned *abort_flag, int lane) {
    const int nseg = (P.H + P.seg_rows - 1) / P.seg_rows;
    const int g = seg + lane / 3 - 1, s = strip + lane % 3 - 1;
    const bool mine = lane < 9 && g >= 0 && g < nseg && s >= 0 && s < P.nstrips;
    return warp_wait_ge(mine ? P.progress + (size_t)g * P.nstrips + s : nullptr, need, abort_flag,
                        kWaitPolls, lane);
}

// Self-test of the failure path: one warp runs the batched kernel's bounded wait with lane 0
// watching a flag that no code ever sets; the wait gives up and reports HS_ERR_TIMEOUT through
// the status word, and the kernel returns (the context stays usable).
__device__ unsigned g_never_set_flag = 0;
__device__ unsigned g_selftest_abort = 0;

__global__ void wait_selftest_kernel(int *status, unsigned long long max_polls) {
    const int lane = threadIdx.x & 31;
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;  // one whole warp
    if (!warp_wait_ge(lane == 0 ? &g_never_set_flag : nullptr, 1u, &g_selftest_abort, max_polls, lane))
        if (lane == 0) atomicCAS(status, 0, (int)HS_ERR_TIMEOUT);
}

// (pass, pair, local tile) of work item `g`: the last unit whose first item is <= g.
__device__ __forceinline__ void decode(const BatchParams &bp, int g, int &pass, int &pair, int &local) {
    int lo = 0, hi = bp.nunits - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(bp.unit_first + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    const int pp = __ldg(bp.unit_pp + lo);
    pass = pp >> 8;
    pair = pp & 255;
    local = g - __ldg(bp.unit_first + lo);
}

template <int T, bool WIDE>
constexpr int batch_min_blocks() { return WIDE ? (T <= 4 ? 3 : 2) : (T <= 4 ? 4 : (T <= 6 ? 3 : 2)); }
template <int T, bool WIDE>
constexpr int batch_warp_floats() { return WIDE ? GeoW<T>::warp_floats : Geo<T>::warp_floats; }
template <int T, bool WIDE>
constexpr int batch_smem() { return WIDE ? GeoW<T>::smem_bytes : Geo<T>::smem_bytes; }

// WIDE: the fast form in the 4-columns-per-lane layout (128-column tiles).
template <int T, bool FAST, bool WIDE>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (batch_min_blocks<T, WIDE>()))
    hs_batch_kernel(const __grid_constant__ BatchParams bp) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *wbase = reinterpret_cast<float *>(smem4) + warp * batch_warp_floats<T, WIDE>();

    griddep_launch_dependents();
    griddep_wait();

    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(bp.queue, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= bp.total_items) break;
        int pass, pi, local;
        decode(bp, g, pass, pi, local);
        const BatchPair &P = bp.pair[pi];
        const int strip = local % P.nstrips;
        const int seg = local / P.nstrips;
        int ok = 1;
        if (lane == 0) ok = (*(volatile const unsigned *)bp.abort_flag == 0);
        ok = __shfl_sync(kFull, ok, 0);
        if (ok && pass > 0) ok = wait_neighbours(P, seg, strip, (unsigned)pass, bp.abort_flag, lane);
        if (!ok) {
            if (lane == 0) {
                atomicCAS(bp.status, 0, (int)HS_ERR_TIMEOUT);
                atomicExch(bp.abort_flag, 1u);
            }
            break;
        }
        __syncwarp();

        SweepParams sp;
        const int src = (P.start + pass) & 1;
        sp.Ix = P.Ix;
        sp.Iy = P.Iy;
        sp.It = P.It;
        sp.u_in = P.U[src];
        sp.v_in = P.V[src];
        sp.u_out = P.U[src ^ 1];
        sp.v_out = P.V[src ^ 1];
        sp.H = P.H;
        sp.W = P.W;
        sp.ld = P.ld;
        sp.alpha2 = P.alpha2;
        sp.alpha_dev = nullptr;
        sp.dump = 0;
        sp.we = bp.we;
        sp.wc = bp.wc;
        sp.seg_rows = P.seg_rows;
        sp.nstrips = P.nstrips;
        sp.nitems = P.items;
        if constexpr (WIDE) {
            ItemW it;
            init_item_w<T>(it, sp, strip, seg, lane, wbase);
            run_item_w<T>(sp, it);
        } else {
            Item it;
            init_item<T>(it, sp, strip, seg, lane, wbase);
            run_item<T, FAST>(sp, it);
        }

        // every lane makes its own stores visible GPU-wide before the warp publishes
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(P.progress + (size_t)seg * P.nstrips + strip, (unsigned)(pass + 1));
    }
}

// ------------------------------------------------------------------ host side

struct PairPlan {
    int idx;  // position in the caller's array
    int H, W, ld, iters, passes, rem, start, nstrips, seg_rows, nseg, items;
    bool wide;
    size_t off_planes, off_progress;
};

static int batch_seg_rows(int H, int T, int cfg_rows) {
    if (cfg_rows > 0) return std::max(std::min(cfg_rows, H), std::min(H, T));
    return std::min(H, std::max(96, T));
}

static hs_status plan_batch(const hs_pair_desc *pairs, int n, const hs_config *cfg,
                            ResolvedConfig &rc, std::vector<PairPlan> &plan, size_t &total,
                            size_t &order_off) {
    hs_status st = resolve_config(cfg, &rc);
    if (st != HS_OK) return st;
    if (!pairs) HS_FAIL(HS_ERR_INVALID_ARG, "pairs is NULL");
    if (n < 1 || n > kMaxBatch) HS_FAIL(HS_ERR_INVALID_ARG, "n=%d outside 1..%d", n, kMaxBatch);
    const int T = rc.T;
    plan.clear();
    size_t off = kHeaderBytes;
    for (int i = 0; i < n; ++i) {
        const hs_pair_desc &d = pairs[i];
        if ((st = check_plane_geometry(d.H, d.W, d.ld)) != HS_OK) return st;
        if (d.iters < 0) HS_FAIL(HS_ERR_INVALID_ARG, "pair %d: iters=%d < 0", i, d.iters);
        if (d.reserved != 0) HS_FAIL(HS_ERR_INVALID_ARG, "pair %d: reserved must be zero", i);
        PairPlan p;
        p.idx = i;
        p.H = d.H;
        p.W = d.W;
        p.ld = d.ld;
        p.iters = d.iters;
        p.passes = d.iters / T;
        p.rem = d.iters % T;
        const int total_passes = p.passes + (p.rem ? 1 : 0);
        p.start = total_passes & 1;  // the last pass writes buffer 0, the caller's u, v
        // 4 columns per lane only when asked for (hs_config.layout = 2): in a persistent
        // launch a tile's latency bounds the chain of dependent passes, and the wider tiles
        // take twice as long (measured: the mixed 64-pair batch at T = 6 runs 37 ms with 2
        // columns per lane, 61 ms with 4, 101 ms with each pair in its size's layout)
        p.wide = rc.fast && rc.layout == 2;
        const int sc = p.wide ? strip_cols_wide(T) : strip_cols_for(T);
        p.nstrips = (d.W + sc - 1) / sc;
        p.seg_rows = batch_seg_rows(d.H, T, rc.seg_rows);
        p.nseg = (d.H + p.seg_rows - 1) / p.seg_rows;
        p.items = p.nstrips * p.nseg;
        p.off_planes = off;
        off += 5 * round_up(plane_bytes(d.H, d.ld), 256);
        plan.push_back(p);
    }
    for (auto &p : plan) {
        p.off_progress = off;
        off += round_up(sizeof(unsigned) * (size_t)p.items, 16);
    }
    // the unit tables of the two launches (pairs of one layout each): at most one unit per
    // full pass of every pair, plus one end entry per launch
    long units = 0;
    for (const auto &p : plan) units += p.passes;
    if (units > (1L << 26)) HS_FAIL(HS_ERR_UNSUPPORTED, "batch has %ld passes in all", units);
    off = round_up(off, 256);
    order_off = off;
    off += round_up(sizeof(int) * (size_t)(2 * units + 2), 256);
    total = round_up(off, 256);
    return HS_OK;
}

template <int T, bool FAST, bool WIDE>
static hs_status launch_batch(const BatchParams &bp, cudaStream_t stream) {
    auto fn = hs_batch_kernel<T, FAST, WIDE>;
    constexpr int smem = batch_smem<T, WIDE>();
    static std::mutex mu;
    static int blocks_per_sm[64] = {};
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    int bps = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev < 64 && blocks_per_sm[dev] == 0) {
            HS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            int b = 0;
            HS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kWarpsPerBlock * 32, smem));
            blocks_per_sm[dev] = std::max(b, 1);
        }
        bps = dev < 64 ? blocks_per_sm[dev] : 1;
    }
    const long want = (long)sm_count() * bps;
    const long need = ((long)bp.total_items + kWarpsPerBlock - 1) / kWarpsPerBlock;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)std::max(1L, std::min(want, need)));
    cfg.blockDim = dim3(kWarpsPerBlock * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HS_CUDA_CHECK(cudaLaunchKernelEx(&cfg, fn, bp));
    return HS_OK;
}

static hs_status launch_batch_any(int T, bool fast, bool wide, const BatchParams &bp, cudaStream_t s) {
#define HS_CASE(TT)                                                                  \
    case TT:                                                                         \
        return wide ? launch_batch<TT, true, true>(bp, s)                            \
                    : (fast ? launch_batch<TT, true, false>(bp, s) : launch_batch<TT, false, false>(bp, s));
    switch (T) {
        HS_CASE(1) HS_CASE(2) HS_CASE(3) HS_CASE(4) HS_CASE(5) HS_CASE(6) HS_CASE(7) HS_CASE(8)
    }
#undef HS_CASE
    HS_FAIL(HS_ERR_INVALID_ARG, "sweeps_per_pass=%d outside 1..%d", T, HS_MAX_SWEEPS_PER_PASS);
}

}  // namespace hs

using namespace hs;

extern "C" {

size_t hs_forward_batched_workspace_bytes(const hs_pair_desc *pairs, int n, const hs_config *cfg) {
    ResolvedConfig rc;
    std::vector<PairPlan> plan;
    size_t total = 0, order_off = 0;
    if (plan_batch(pairs, n, cfg, rc, plan, total, order_off) != HS_OK) return 0;
    return total;
}

hs_status hs_forward_batched(const hs_pair_desc *pairs, int n, void *workspace,
                             size_t workspace_bytes, const hs_config *cfg, int *device_status,
                             void *stream) {
    clear_error();
    ResolvedConfig rc;
    std::vector<PairPlan> plan;
    size_t total = 0, order_off = 0;
    hs_status st = plan_batch(pairs, n, cfg, rc, plan, total, order_off);
    if (st != HS_OK) return st;
    if (!workspace || workspace_bytes < total)
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, total);
    if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
        HS_FAIL(HS_ERR_ALIGNMENT, "workspace is not 256-byte aligned");
    for (int i = 0; i < n; ++i) {
        const hs_pair_desc &d = pairs[i];
        const void *pl[4] = {d.I0, d.I1, d.u, d.v};
        const char *nm[4] = {"I0", "I1", "u", "v"};
        for (int k = 0; k < 4; ++k)
            if ((st = check_plane(pl[k], nm[k])) != HS_OK) {
                set_error("pair %d: %s", i, hs_last_error());
                return st;
            }
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *ws = reinterpret_cast<char *>(workspace);
    int *status = device_status ? device_status : reinterpret_cast<int *>(ws + 4);
    unsigned *abort_flag = reinterpret_cast<unsigned *>(ws + 8);

    // header and every pair's tile-progress counters start at zero
    HS_CUDA_CHECK(cudaMemsetAsync(ws, 0, kHeaderBytes, s));
    if (device_status) HS_CUDA_CHECK(cudaMemsetAsync(device_status, 0, sizeof(int), s));
    const size_t prog_begin = plan.front().off_progress;
    HS_CUDA_CHECK(cudaMemsetAsync(ws + prog_begin, 0, total - prog_begin, s));

    // pair buffers
    std::vector<BatchPair> bpairs(n);
    DerivParams dp;
    memset(&dp, 0, sizeof(dp));
    dp.npairs = n;
    int maxW = 1, maxH = 1;
    for (int i = 0; i < n; ++i) {
        const PairPlan &p = plan[i];
        const hs_pair_desc &d = pairs[i];
        const size_t pb = round_up(plane_bytes(p.H, p.ld), 256);
        float *base = reinterpret_cast<float *>(ws + p.off_planes);
        BatchPair &b = bpairs[i];
        b.Ix = base;
        b.Iy = reinterpret_cast<float *>(ws + p.off_planes + pb);
        b.It = reinterpret_cast<float *>(ws + p.off_planes + 2 * pb);
        b.U[0] = d.u;
        b.V[0] = d.v;
        b.U[1] = reinterpret_cast<float *>(ws + p.off_planes + 3 * pb);
        b.V[1] = reinterpret_cast<float *>(ws + p.off_planes + 4 * pb);
        b.progress = reinterpret_cast<unsigned *>(ws + p.off_progress);
        b.H = p.H;
        b.W = p.W;
        b.ld = p.ld;
        b.alpha2 = d.alpha * d.alpha;
        b.passes = p.passes;
        b.start = p.start;
        b.nstrips = p.nstrips;
        b.seg_rows = p.seg_rows;
        b.items = p.items;
        dp.I0[i] = d.I0;
        dp.I1[i] = d.I1;
        dp.Ix[i] = const_cast<float *>(b.Ix);
        dp.Iy[i] = const_cast<float *>(b.Iy);
        dp.It[i] = const_cast<float *>(b.It);
        dp.U0[i] = b.U[p.start];
        dp.V0[i] = b.V[p.start];
        dp.H[i] = p.H;
        dp.W[i] = p.W;
        dp.ld[i] = p.ld;
        maxW = std::max(maxW, p.W);
        maxH = std::max(maxH, p.H);
    }
    {
        dim3 block(64, 4);
        dim3 grid((unsigned)((maxW + 63) / 64), (unsigned)((maxH + 3) / 4), (unsigned)n);
        batch_derivs_kernel<<<grid, block, 0, s>>>(dp);
        HS_LAUNCH_CHECK("batch_derivs_kernel");
    }

    // persistent kernels over every full pass of every pair: one launch per layout
    int *order = reinterpret_cast<int *>(ws + order_off);
    for (int lay = 1; lay >= 0; --lay) {
        const bool wide = lay == 1;
        std::vector<int> members;
        for (int i = 0; i < n; ++i)
            if (plan[i].wide == wide && bpairs[i].passes > 0) members.push_back(i);
        if (members.empty()) continue;
        const int m = (int)members.size();
        BatchParams bp;
        memset(&bp, 0, sizeof(bp));
        bp.npairs = m;
        bp.we = rc.we;
        bp.wc = rc.wc;
        bp.queue = reinterpret_cast<unsigned *>(ws + (wide ? 12 : 0));
        bp.status = status;
        bp.abort_flag = abort_flag;
        long total_items = 0;
        bp.unit_prefix[0] = 0;
        for (int r = 0; r < m; ++r) {
            bp.pair[r] = bpairs[members[r]];
            bp.unit_prefix[r + 1] = bp.unit_prefix[r] + bp.pair[r].passes;
            total_items += (long)bp.pair[r].passes * bp.pair[r].items;
        }
        if (total_items > 0x7fffffffL) HS_FAIL(HS_ERR_UNSUPPORTED, "batch has too many work items");
        bp.nunits = bp.unit_prefix[m];
        bp.total_items = (int)total_items;
        bp.unit_pp = order;
        bp.unit_first = order + bp.nunits;
        order += 2 * bp.nunits + 1;
        batch_order_kernel<<<1, 1024, 0, s>>>(bp);
        HS_LAUNCH_CHECK("batch_order_kernel");
        if ((st = launch_batch_any(rc.T, rc.fast, wide, bp, s)) != HS_OK) return st;
    }

    // the short last pass of pairs whose sweep count is not a multiple of T
    for (int i = 0; i < n; ++i) {
        const PairPlan &p = plan[i];
        if (p.rem == 0) continue;
        const BatchPair &b = bpairs[i];
        const int src = (p.start + p.passes) & 1;
        SweepParams pp;
        pp.Ix = b.Ix;
        pp.Iy = b.Iy;
        pp.It = b.It;
        pp.u_in = b.U[src];
        pp.v_in = b.V[src];
        pp.u_out = b.U[src ^ 1];
        pp.v_out = b.V[src ^ 1];
        pp.H = p.H;
        pp.W = p.W;
        pp.ld = p.ld;
        pp.alpha2 = b.alpha2;
        pp.alpha_dev = nullptr;
        pp.dump = 0;
        pp.we = rc.we;
        pp.wc = rc.wc;
        const int sc = strip_cols_for(p.rem);
        pp.nstrips = (p.W + sc - 1) / sc;
        pp.seg_rows = default_seg_rows(p.H, pp.nstrips, p.rem);
        pp.nitems = pp.nstrips * ((p.H + pp.seg_rows - 1) / pp.seg_rows);
        if ((st = launch_pass(p.rem, rc.fast, pp, s)) != HS_OK) return st;
    }
    return HS_OK;
}

hs_status hs_selftest_bounded_wait(int *device_status, int max_polls, void *stream) {
    clear_error();
    if (!device_status) HS_FAIL(HS_ERR_INVALID_ARG, "device_status is NULL");
    if (max_polls < 1 || (unsigned long long)max_polls > kWaitPolls)
        HS_FAIL(HS_ERR_INVALID_ARG, "max_polls=%d outside 1..%llu", max_polls, kWaitPolls);
    wait_selftest_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(device_status, (unsigned long long)max_polls);
    HS_LAUNCH_CHECK("wait_selftest_kernel");
    return HS_OK;
}

}  // extern "C"
