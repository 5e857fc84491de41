// hs_stream4.cuh -- the wide form of the streaming Horn-Schunck sweep for the fast
// arithmetic mode: 4 adjacent columns per lane, a 128-column strip per warp.
//
// Same pipeline as hs_stream.cuh (T sweeps per HBM pass as a register pipeline down the
// strip, rolling 2-register windows per column-plane, a per-warp shared-memory ring fed
// by cp.async, a (T+1)-slot ring of packed coefficients), with three differences that cut
// the instructions per cell-sweep:
//   - a lane's 4 columns are one 16-byte chunk of each plane row, which the lane copies and
//     reads itself: no lane reads another's copy, so no warp barrier brackets the copy;
//   - per stage and plane only the two lane-edge columns cross lanes (one shuffle each
//     way for 4 cells instead of 2);
//   - the per-step bookkeeping (copies, ring indices, stores) is spread over twice the
//     cells, and the temporal halo (T rounded up to 4 columns each side) is a smaller share
//     of the strip (120 or 112 output columns of 128).
// Only the fast form (FMA, reciprocal of the denominator) exists in this layout; the exact
// form keeps the 2-column layout, whose tap-ordered windows need 5 registers per column.
#pragma once

#include "hs_stream.cuh"

namespace hs {

constexpr int kWideCols = 128;        // columns per strip (4 per lane)
constexpr int kWidePrefetch = 2;      // rows in flight per warp
constexpr int kWideRawSlots = kWidePrefetch + 1;

template <int T>
struct GeoW {
    static constexpr int halo = (T + 3) & ~3;                  // 16-byte aligned lane chunks
    static constexpr int strip = kWideCols - 2 * halo;         // output columns per strip
    static constexpr int coef_slots = T + 1;                   // rows k-T .. k
    static constexpr int raw_floats = kWideRawSlots * kRawPlanes * kWideCols;
    static constexpr int coef_floats = coef_slots * 4 * 32 * 4;  // [slot][column][lane] float4
    static constexpr int warp_floats = raw_floats + coef_floats;
    static constexpr int smem_bytes = kWarpsPerBlock * warp_floats * (int)sizeof(float);
};

struct ItemW {
    float *raw;     // [kWideRawSlots][kRawPlanes][128]
    float4 *coef;   // [T+1][4][32]
    int lane;
    int lcol;       // this lane's chunk, clamped to an in-bounds chunk of the row
    int xa;         // first of the lane's 4 columns
    unsigned last;  // bit j: column xa+j is W-1 (right neighbour is itself)
    unsigned st;    // bit j: column xa+j is an output of this strip
    bool first;     // column xa is 0 (left neighbour is itself)
    int y_start, y_end;
    float alpha2;
};

__device__ __forceinline__ void issue_row_w(const ItemW &it, int slot, int row, const SweepParams &p) {
    row = min(max(row, 0), p.H - 1);
    const size_t off = (size_t)row * p.ld + it.lcol;
    float *base = it.raw + slot * (kRawPlanes * kWideCols) + 4 * it.lane;
    cp_async16(base + 0 * kWideCols, p.u_in + off);
    cp_async16(base + 1 * kWideCols, p.v_in + off);
    cp_async16(base + 2 * kWideCols, p.Ix + off);
    cp_async16(base + 3 * kWideCols, p.Iy + off);
    cp_async16(base + 4 * kWideCols, p.It + off);
    cp_async_commit();
}

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

template <int T, bool XEDGE, bool EDGE>
__device__ __forceinline__ void stream_step_w(const SweepParams &p, const ItemW &it,
                                              Win<true> (&w)[T][2][4], int k, int rslot, int cslot) {
    // prefetch row k + kWidePrefetch into the slot row k-1 used, then wait for row k; the
    // lane only ever reads its own copies
    issue_row_w(it, rslot == 0 ? kWideRawSlots - 1 : rslot - 1, min(k + kWidePrefetch, it.y_end - 1 + T), p);
    cp_async_wait<kWidePrefetch>();

    // stage 0: unpack row k; pack its coefficients with the reciprocal denominator
    const float *raw = it.raw + rslot * (kRawPlanes * kWideCols) + 4 * it.lane;
    const float4 u4 = lds4(raw), v4 = lds4(raw + kWideCols);
    {
        const float4 ix = lds4(raw + 2 * kWideCols), iy = lds4(raw + 3 * kWideCols);
        const float4 t4 = lds4(raw + 4 * kWideCols);
        float4 *cs = it.coef + cslot * 128 + it.lane;
        cs[0] = make_float4(ix.x, iy.x, t4.x, rcp_approx(fmaf(iy.x, iy.x, fmaf(ix.x, ix.x, it.alpha2))));
        cs[32] = make_float4(ix.y, iy.y, t4.y, rcp_approx(fmaf(iy.y, iy.y, fmaf(ix.y, ix.y, it.alpha2))));
        cs[64] = make_float4(ix.z, iy.z, t4.z, rcp_approx(fmaf(iy.z, iy.z, fmaf(ix.z, ix.z, it.alpha2))));
        cs[96] = make_float4(ix.w, iy.w, t4.w, rcp_approx(fmaf(iy.w, iy.w, fmaf(ix.w, ix.w, it.alpha2))));
    }
    float cu[2][4] = {{u4.x, u4.y, u4.z, u4.w}, {v4.x, v4.y, v4.z, v4.w}};  // [plane][column]

#pragma unroll
    for (int s = 0; s < T; ++s) {
        const int n = k - s;  // arriving row (input of sweep s+1)
        float ub[2][4];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float c0 = cu[q][0], c1 = cu[q][1], c2 = cu[q][2], c3 = cu[q][3];
            float l0 = __shfl_up_sync(kFull, c3, 1);
            float r3 = __shfl_down_sync(kFull, c0, 1);
            float r0 = c1, r1 = c2, r2 = c3;
            if constexpr (XEDGE) {
                l0 = it.first ? c0 : l0;
                r0 = (it.last & 1u) ? c0 : r0;
                r1 = (it.last & 2u) ? c1 : r1;
                r2 = (it.last & 4u) ? c2 : r2;
                r3 = (it.last & 8u) ? c3 : r3;
            }
            ub[q][0] = win_step<EDGE>(w[s][q][0], l0, c0, r0, n, p.H, p.we, p.wc);
            ub[q][1] = win_step<EDGE>(w[s][q][1], c0, c1, r1, n, p.H, p.we, p.wc);
            ub[q][2] = win_step<EDGE>(w[s][q][2], c1, c2, r2, n, p.H, p.we, p.wc);
            ub[q][3] = win_step<EDGE>(w[s][q][3], c2, c3, r3, n, p.H, p.we, p.wc);
        }
        int rs = cslot - (s + 1);
        if (rs < 0) rs += GeoW<T>::coef_slots;
        const float4 *cr = it.coef + rs * 128 + it.lane;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float4 C = cr[32 * j];
            const float ubar = ub[0][j], vbar = ub[1][j];
            const float t = fmaf(C.x, ubar, fmaf(C.y, vbar, C.z)) * C.w;
            cu[0][j] = fmaf(-C.x, t, ubar);
            cu[1][j] = fmaf(-C.y, t, vbar);
        }
    }

    // store sweep T of row k - T
    const int r = k - T;
    if (r >= it.y_start && r < it.y_end) {
        const size_t off = (size_t)r * p.ld + it.xa;
        if (it.st == 15u) {
            *reinterpret_cast<float4 *>(p.u_out + off) = make_float4(cu[0][0], cu[0][1], cu[0][2], cu[0][3]);
            *reinterpret_cast<float4 *>(p.v_out + off) = make_float4(cu[1][0], cu[1][1], cu[1][2], cu[1][3]);
        } else if (it.st) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (it.st & (1u << j)) {
                    p.u_out[off + j] = cu[0][j];
                    p.v_out[off + j] = cu[1][j];
                }
        }
    }
}

template <int T, bool XEDGE>
__device__ __forceinline__ void stream_item_w(const SweepParams &p, const ItemW &it) {
    const int k0 = max(0, it.y_start - T);
    const int k_end = it.y_end - 1 + T;
    Win<true> w[T][2][4];
#pragma unroll
    for (int s = 0; s < T; ++s)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int j = 0; j < 4; ++j) w[s][q][j] = Win<true>{};

#pragma unroll
    for (int i = 0; i < kWidePrefetch; ++i) issue_row_w(it, i, k0 + i, p);

    // steps in [klo, khi] have no stage at row 0 or past row H-2: no clamp logic
    const int klo = max(k0, T);
    const int khi = min(k_end, p.H - 2);
    int k = k0, rslot = 0, cslot = 0;
    auto advance = [&]() {
        ++k;
        rslot = (rslot + 1 == kWideRawSlots) ? 0 : rslot + 1;
        cslot = (cslot + 1 == GeoW<T>::coef_slots) ? 0 : cslot + 1;
    };
    if (klo + 1 <= khi) {
        for (; k < klo; advance()) stream_step_w<T, XEDGE, true>(p, it, w, k, rslot, cslot);
        while (k + 1 <= khi) {
            stream_step_w<T, XEDGE, false>(p, it, w, k, rslot, cslot);
            advance();
            stream_step_w<T, XEDGE, false>(p, it, w, k, rslot, cslot);
            advance();
        }
    }
    for (; k <= k_end; advance()) stream_step_w<T, XEDGE, true>(p, it, w, k, rslot, cslot);
    cp_async_wait<0>();
}

template <int T>
__device__ __forceinline__ void init_item_w(ItemW &it, const SweepParams &p, int strip, int seg,
                                            int lane, float *wbase) {
    using G = GeoW<T>;
    const int x0 = strip * G::strip - G::halo;  // a multiple of 4
    it.raw = wbase;
    it.coef = reinterpret_cast<float4 *>(wbase + G::raw_floats);
    it.lane = lane;
    it.xa = x0 + 4 * lane;
    // a chunk lies wholly inside or outside the row (xa and ld are multiples of 4); outside
    // ones copy any in-bounds chunk (their columns never feed a stored pixel)
    it.lcol = (it.xa >= 0 && it.xa + 4 <= p.ld) ? it.xa : 0;
    it.first = (it.xa == 0);
    const int vlo = strip * G::strip, vhi = min(vlo + G::strip, p.W);
    it.last = 0u;
    it.st = 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int x = it.xa + j;
        if (x == p.W - 1) it.last |= 1u << j;
        if (x >= vlo && x < vhi) it.st |= 1u << j;
    }
    it.y_start = seg * p.seg_rows;
    it.y_end = min(p.H, it.y_start + p.seg_rows);
    it.alpha2 = p.alpha_dev ? __fmul_rn(__ldg(p.alpha_dev), __ldg(p.alpha_dev)) : p.alpha2;
}

template <int T>
__device__ __forceinline__ void run_item_w(const SweepParams &p, const ItemW &it) {
    const int x0 = it.xa - 4 * it.lane;
    if (x0 <= 0 || x0 + kWideCols >= p.W) stream_item_w<T, true>(p, it);
    else stream_item_w<T, false>(p, it);
}

int strip_cols_wide(int T);

}  // namespace hs
