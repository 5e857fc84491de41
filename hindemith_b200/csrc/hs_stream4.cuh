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
// The arithmetic runs on column pairs (0, 1) and (2, 3) with the sm_100 packed FP32
// instructions (one instruction, two IEEE operations rounded as their scalar forms).  The
// pairs are the halves of the lane's 16-byte chunk as loaded, the coefficient ring holds each
// coefficient's 4 columns as loaded (Ix, Iy, It and -1/den), and the horizontal neighbour
// sums left + right are formed as scalar adds straight into their pair: no value is moved
// to repack a pair.  The update is then three packed FMAs and one packed multiply per pair;
// results equal the scalar 2-column kernel's bit for bit.  Only the fast form (FMA, reciprocal of the denominator) exists in this layout; the
// exact form keeps the 2-column layout, whose tap-ordered windows need 5 registers per column.
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
    static constexpr int coef_floats = coef_slots * 4 * 32 * 4;  // [slot][coef][lane] float4
    static constexpr int warp_floats = raw_floats + coef_floats;
    static constexpr int smem_bytes = kWarpsPerBlock * warp_floats * (int)sizeof(float);
};

struct ItemW {
    float *raw;     // [kWideRawSlots][kRawPlanes][128]
    float4 *coef;   // [T+1][4][32]: Ix, Iy, It, -1/den of the lane's 4 columns
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

// HEAD: one of the first 2T-2 steps of a segment that starts T or more rows below the
// image top; stage s only runs from its segment step kk = k - k0 = 2s on (see stream_item_w).
// XE: 0 = no image side in the strip; 1 = a side, any W; 2 = a side with W % 4 == 0, where
// column W-1 is always a lane's last column (chunks start at multiples of 4), so only the
// first column's left clamp and the last column's right clamp can apply.
// DUMP (the training recompute) also writes every stage's sweep to p.dump_u/v.
template <int T, int XE, bool EDGE, bool HEAD = false, bool DUMP = false>
__device__ __forceinline__ void stream_step_w(const SweepParams &p, const ItemW &it,
                                              Win<true> (&w)[T][2][2], int k, int rslot, int cslot,
                                              int kk = 0) {
    // prefetch row k + kWidePrefetch into the slot row k-1 used, then wait for row k; the
    // lane only ever reads its own copies
    issue_row_w(it, rslot == 0 ? kWideRawSlots - 1 : rslot - 1, min(k + kWidePrefetch, it.y_end - 1 + T), p);
    cp_async_wait<kWidePrefetch>();

    // stage 0: unpack row k; keep its coefficients as loaded, with -1/den
    const float *raw = it.raw + rslot * (kRawPlanes * kWideCols) + 4 * it.lane;
    const float4 u4 = lds4(raw), v4 = lds4(raw + kWideCols);
    {
        const float4 ix = lds4(raw + 2 * kWideCols), iy = lds4(raw + 3 * kWideCols);
        const float4 t4 = lds4(raw + 4 * kWideCols);
        float4 nw;
        nw.x = -rcp_approx(fmaf(iy.x, iy.x, fmaf(ix.x, ix.x, it.alpha2)));
        nw.y = -rcp_approx(fmaf(iy.y, iy.y, fmaf(ix.y, ix.y, it.alpha2)));
        nw.z = -rcp_approx(fmaf(iy.z, iy.z, fmaf(ix.z, ix.z, it.alpha2)));
        nw.w = -rcp_approx(fmaf(iy.w, iy.w, fmaf(ix.w, ix.w, it.alpha2)));
        float4 *cs = it.coef + cslot * 128 + it.lane;
        cs[0] = ix;
        cs[32] = iy;
        cs[64] = t4;
        cs[96] = nw;
    }
    // [plane][pair]: pair 0 holds columns (0, 1), pair 1 columns (2, 3)
    float2 cu[2][2] = {{make_float2(u4.x, u4.y), make_float2(u4.z, u4.w)},
                       {make_float2(v4.x, v4.y), make_float2(v4.z, v4.w)}};
    const float2 we2 = make_float2(p.we, p.we), wc2 = make_float2(p.wc, p.wc);

#pragma unroll
    for (int s = 0; s < T; ++s) {
        if (HEAD && kk < 2 * s) break;  // warp-uniform; later stages start later still
        const int n = k - s;  // arriving row (input of sweep s+1)
        float2 ub[2][2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float2 E = cu[q][0], O = cu[q][1];  // (c0, c1), (c2, c3)
            const float lsh = __shfl_up_sync(kFull, O.y, 1);    // column -1: lane-1's c3
            const float rsh = __shfl_down_sync(kFull, E.x, 1);  // column 4: lane+1's c0
            // left and right neighbours: the column itself at an image side
            float L0 = lsh, R0 = E.y, R1 = O.x, R2 = O.y, R3 = rsh;
            if constexpr (XE == 1) {
                L0 = it.first ? E.x : L0;
                R0 = (it.last & 1u) ? E.x : R0;
                R1 = (it.last & 2u) ? E.y : R1;
                R2 = (it.last & 4u) ? O.x : R2;
                R3 = (it.last & 8u) ? O.y : R3;
            } else if constexpr (XE == 2) {
                L0 = it.first ? E.x : L0;
                R3 = (it.last & 8u) ? O.y : R3;
            }
            const float2 hE = make_float2(__fadd_rn(L0, R0), __fadd_rn(E.x, R1));
            const float2 hO = make_float2(__fadd_rn(E.y, R2), __fadd_rn(O.x, R3));
            ub[q][0] = win_step_h<EDGE>(w[s][q][0], hE, E, n, p.H, we2, wc2);
            ub[q][1] = win_step_h<EDGE>(w[s][q][1], hO, O, n, p.H, we2, wc2);
        }
        int rs = cslot - (s + 1);
        if (rs < 0) rs += GeoW<T>::coef_slots;
        const float4 *cr = it.coef + rs * 128 + it.lane;
        const float4 cX = cr[0], cY = cr[32], cT = cr[64], cN = cr[96];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float2 cx = j ? make_float2(cX.z, cX.w) : make_float2(cX.x, cX.y);
            const float2 cy = j ? make_float2(cY.z, cY.w) : make_float2(cY.x, cY.y);
            const float2 ct = j ? make_float2(cT.z, cT.w) : make_float2(cT.x, cT.y);
            const float2 nw = j ? make_float2(cN.z, cN.w) : make_float2(cN.x, cN.y);
            const float2 ubar = ub[0][j], vbar = ub[1][j];
            // -t = (Ix ubar + Iy vbar + It) * (-1/den); u = ubar + Ix (-t) = ubar - Ix t
            const float2 nt = mul2(fma2(cx, ubar, fma2(cy, vbar, ct)), nw);
            cu[0][j] = fma2(cx, nt, ubar);
            cu[1][j] = fma2(cy, nt, vbar);
        }
        if constexpr (DUMP) {  // write sweep s+1 of row k-s-1 (state dumps)
            const int rr = k - s - 1;
            if (rr >= it.y_start && rr < it.y_end) {
                const size_t off = (size_t)rr * p.ld + it.xa;
                const float du[4] = {cu[0][0].x, cu[0][0].y, cu[0][1].x, cu[0][1].y};
                const float dv[4] = {cu[1][0].x, cu[1][0].y, cu[1][1].x, cu[1][1].y};
                if (it.st == 15u) {
                    *reinterpret_cast<float4 *>(p.dump_u[s] + off) = make_float4(du[0], du[1], du[2], du[3]);
                    *reinterpret_cast<float4 *>(p.dump_v[s] + off) = make_float4(dv[0], dv[1], dv[2], dv[3]);
                } else if (it.st) {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (it.st & (1u << j)) {
                            p.dump_u[s][off + j] = du[j];
                            p.dump_v[s][off + j] = dv[j];
                        }
                }
            }
        }
    }

    // store sweep T of row k - T
    const int r = k - T;
    if (r >= it.y_start && r < it.y_end) {
        const size_t off = (size_t)r * p.ld + it.xa;
        const float uo[4] = {cu[0][0].x, cu[0][0].y, cu[0][1].x, cu[0][1].y};
        const float vo[4] = {cu[1][0].x, cu[1][0].y, cu[1][1].x, cu[1][1].y};
        if (it.st == 15u) {
            *reinterpret_cast<float4 *>(p.u_out + off) = make_float4(uo[0], uo[1], uo[2], uo[3]);
            *reinterpret_cast<float4 *>(p.v_out + off) = make_float4(vo[0], vo[1], vo[2], vo[3]);
        } else if (it.st) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (it.st & (1u << j)) {
                    p.u_out[off + j] = uo[j];
                    p.v_out[off + j] = vo[j];
                }
        }
    }
}

// UNR: the main loop body holds two steps.  The rolled loop is shorter code; with one-warp
// CTAs on an L2-resident image, where
// instruction fetch is the leading stall, it measured faster (1080p T = 6: 511 against 500
// Gpix-it/s), the unrolled one on images larger than L2 (4096^2 T = 5: 822 against 805).
template <int T, int XE, bool DUMP, bool UNR = true>
__device__ __forceinline__ void stream_item_w(const SweepParams &p, const ItemW &it) {
    const int k0 = max(0, it.y_start - T);
    const int k_end = it.y_end - 1 + T;
    Win<true> w[T][2][2];
#pragma unroll
    for (int s = 0; s < T; ++s)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int j = 0; j < 2; ++j) w[s][q][j] = Win<true>{};

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
    // A segment starting T or more rows below the top (k0 = y_start - T > 0) needs stage s's
    // output only from row y_start - (T-1-s) = k0 + s + 1 on, which it first emits at
    // segment step 2s + 2, from the rows it receives at steps 2s and 2s + 1 (stage s-1's
    // first valid rows).  Stage s therefore does nothing useful before step 2s: the first
    // 2T-2 steps skip those stages, T(T-1) stage-steps per segment.
    if (!DUMP && k0 >= T && k0 + 2 * T - 2 <= khi) {  // (dump passes: as the 2-column kernel)
        for (int kk = 0; kk < 2 * T - 2; ++kk, advance())
            stream_step_w<T, XE, false, true>(p, it, w, k, rslot, cslot, kk);
    }
    if (klo + 1 <= khi) {
        for (; k < klo; advance()) stream_step_w<T, XE, true, false, DUMP>(p, it, w, k, rslot, cslot);
        if constexpr (UNR) {
            while (k + 1 <= khi) {
                stream_step_w<T, XE, false, false, DUMP>(p, it, w, k, rslot, cslot);
                advance();
                stream_step_w<T, XE, false, false, DUMP>(p, it, w, k, rslot, cslot);
                advance();
            }
        } else {
#pragma unroll 1
            for (; k <= khi; advance()) stream_step_w<T, XE, false, false, DUMP>(p, it, w, k, rslot, cslot);
        }
    }
    for (; k <= k_end; advance()) stream_step_w<T, XE, true, false, DUMP>(p, it, w, k, rslot, cslot);
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

template <int T, bool DUMP = false, bool UNR = true>
__device__ __forceinline__ void run_item_w(const SweepParams &p, const ItemW &it) {
    const int x0 = it.xa - 4 * it.lane;
    if (x0 <= 0 || x0 + kWideCols >= p.W) {
        if ((p.W & 3) == 0) stream_item_w<T, 2, DUMP, UNR>(p, it);
        else stream_item_w<T, 1, DUMP, UNR>(p, it);
    } else {
        stream_item_w<T, 0, DUMP, UNR>(p, it);
    }
}

int strip_cols_wide(int T);

}  // namespace hs
