// hs_stream.cuh -- the streaming, temporally blocked Horn-Schunck sweep (device code
// shared by the per-pass kernel in hs_sweep.cu and the persistent batched kernel in
// hs_batch.cu).
//
// One pass over HBM runs T sweeps.  Each warp owns a work item: a 64-column strip
// (2 adjacent columns per lane) of a segment of rows.  The warp streams the segment's
// rows downward; row k enters stage 0 at step k, and stage s emits sweep s+1 of row
// k-s-1 at the same step, so the T sweeps form a register pipeline down the strip:
//   - horizontal neighbours come from warp shuffles (only the lane-edge column moves),
//   - vertical neighbours come from a rolling window kept in registers (2 values per
//     column and plane in the fast form, tap-ordered accumulators in the exact form),
//   - the rows (u, v, Ix, Iy, It) arrive in a per-warp shared-memory ring through 16-byte
//     cp.async copies three rows ahead; stage 0 repacks the lane's coefficients (Ix, Iy,
//     It and the negated denominator term, each as a column pair) for the stages to read,
//   - the lane's two columns are one packed FP32 pair: the sm_100 f32x2 instructions do
//     both columns' operation in one instruction, each rounded as its scalar form, so the
//     results are those of the scalar operation sequence bit for bit (the exact form's
//     products stay scalar multiplies, which are never fused into the adds).
// A strip loads `halo` extra columns each side (T rounded up to an even count) and
// outputs the middle 64 - 2*halo; a segment starts T rows early; both are the temporal
// blocking halo.  Warps never synchronise with each other; within a warp, a barrier after
// each row's cp.async wait publishes the lanes' copies to the lanes that read them.
//
// Clamp-to-edge boundaries (Stencil2DMVM.cpp:40-47): a neighbour outside the image is
// the pixel itself.  Horizontally the lane substitutes its own value; at the top row 0
// is its own upper neighbour; past the bottom, row H-1 stands in for row H.
//
// Exact mode (FAST = false) reproduces the reference program's FP32 operations one
// rounding at a time in its order: ubar = sum over the 8 taps in row-major order from
// 0; t = ((Ix*ubar + Iy*vbar) + It) / ((alpha2 + Ix*Ix) + Iy*Iy); u = ubar - Ix*t.
// Fast mode factors the average into edge and corner sums, uses fused multiply-adds
// and multiplies by a reciprocal of the denominator computed once per row per pass.
#pragma once

#include "hs_common.cuh"

namespace hs {

constexpr int kWarpCols = 64;                 // columns per strip (2 per lane)
constexpr int kPrefetch = 3;                  // rows in flight per warp
constexpr int kRawSlots = kPrefetch + 1;      // raw-row ring depth (a power of two)
constexpr int kRawPlanes = 5;                 // u, v, Ix, Iy, It as copied from HBM
constexpr int kWarpsPerBlock = 4;             // independent warps per CTA (persistent batch)
// Warps per CTA of the per-pass launches (the plain sweep and the training table and adjoint
// passes).  Each warp is an independent work item, so a one-warp CTA frees its slot the moment
// its item ends: another item, or the next pass's first items under programmatic dependent
// launch, start there at once instead of waiting for the CTA's slowest warp.  The resident
// warps per SM (each kernel's register budget) stay those of 4-warp CTAs.
constexpr int kPassWarps = 1;
constexpr unsigned kFull = 0xffffffffu;

template <int T>
struct Geo {
    static constexpr int halo = (T + 1) & ~1;                  // even: lanes read float2
    // Rows are copied in 16-byte chunks.  A strip starts at x0 = strip*i - halo, which is
    // 16-byte aligned when halo % 4 == 0 ("wide": 16 chunks per plane row); otherwise the
    // copy starts sh = 2 columns early and takes 17 chunks (68 floats) per plane row.
    static constexpr bool wide = (halo % 4) == 0;
    static constexpr int sh = wide ? 0 : 2;
    static constexpr int rw = wide ? kWarpCols : kWarpCols + 4;  // floats per ring plane row
    static constexpr int strip = kWarpCols - 2 * halo;         // output columns per strip
    static constexpr int coef_slots = T + 1;                   // rows k-T .. k
    static constexpr int raw_floats = kRawSlots * kRawPlanes * rw;
    static constexpr int coef_floats = coef_slots * 2 * 32 * 4;  // [slot][2][lane] float4
    static constexpr int warp_floats = raw_floats + coef_floats;
    static constexpr int smem_bytes = kWarpsPerBlock * warp_floats * (int)sizeof(float);
};

struct SweepParams {
    const float *Ix, *Iy, *It;
    const float *u_in, *v_in;
    float *u_out, *v_out;
    int H, W, ld;
    float alpha2;
    const float *alpha_dev;  // if set, alpha2 = alpha_dev[0] squared (device-resident alpha)
    int dump;                // if set, stage s also writes its sweep into dump_u/v[s]
    float *dump_u[HS_MAX_SWEEPS_PER_PASS], *dump_v[HS_MAX_SWEEPS_PER_PASS];
    float we, wc;  // edge and corner weights of the average
    int seg_rows;
    int nstrips;
    int nitems;
};

// 16-byte async copy global -> shared through L2 only (.cg): never served from a stale
// L1 line, so data another CTA wrote during this kernel is seen once it is published.
__device__ __forceinline__ void cp_async16(float *smem, const float *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
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

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

// Sliding three-row window of one stage and one plane, for a pair of columns (the
// vertical recurrences are per column, so two columns run as one packed pair).
//   fast : with Y(k) = we*c(k) + wc*h(k) (h = left + right), the average of row n-1 is
//          Y(n-2) + we*h(n-1) + Y(n).  Z = Y(n-2) + we*h(n-1) and Y1 = Y(n-1) are kept,
//          so a row costs 5 operations and 2 registers per column.
//   exact: A0 = next row's accumulator holding its up taps (taken from row n-1),
//          A1 = row n-1's accumulator holding its up and mid taps, l1/c1/r1 = row n-1
//          (read only for the bottom clamp)
template <bool FAST>
struct Win;
template <>
struct Win<true> {
    float2 Z, Y1;
};
template <>
struct Win<false> {
    float2 A0, A1, l1, c1, r1;
};

// Row n arrives (values l, c, r at the pair's columns); returns the average of row n-1
// and advances the window.  EDGE: the row may be row 0 (top clamp) or past the bottom
// (replaced by row H-1, the bottom clamp).  The fast form has no product feeding an add
// (mul2's restriction).
// The fast form from the row's horizontal neighbour sums hn = left + right.
template <bool EDGE>
__device__ __forceinline__ float2 win_step_h(Win<true> &w, float2 hn, float2 c, int n, int H,
                                             float2 we, float2 wc) {
    float2 yn = fma2(we, c, mul2(wc, hn));
    if (EDGE && n >= H) yn = w.Y1;  // the row below H-1 is row H-1
    const float2 out = add2(w.Z, yn);
    w.Z = fma2(we, hn, (EDGE && n == 0) ? yn : w.Y1);  // row 0's up row is row 0
    w.Y1 = yn;
    return out;
}

template <bool EDGE>
__device__ __forceinline__ float2 win_step(Win<false> &w, float2 l, float2 c, float2 r, int n, int H,
                                           float2 we, float2 wc) {
    if (EDGE && n >= H) { l = w.l1; c = w.c1; r = w.r1; }
    // taps in row-major order: (-1,-1) (0,-1) (1,-1) | (-1,0) (1,0) | (-1,1) (0,1) (1,1)
    const float2 tl = mul2r(wc, l), tc = mul2r(we, c), tr = mul2r(wc, r);
    float2 o = w.A1;                              // row n-1: up and mid taps done
    o = add2(o, tl);                              // its dn taps come from row n
    o = add2(o, tc);
    o = add2(o, tr);
    float2 up = add2(f2(0.0f, 0.0f), tl);         // row n+1's up taps come from row n
    up = add2(up, tc);
    up = add2(up, tr);
    float2 am = (EDGE && n == 0) ? up : w.A0;     // row 0's up taps are its own (clamp)
    am = add2(am, mul2r(we, l));                  // row n's mid taps
    am = add2(am, mul2r(we, r));
    w.A0 = up;
    w.A1 = am;
    if (EDGE) { w.l1 = l; w.c1 = c; w.r1 = r; }
    return o;
}

// Per-warp context of one work item.
struct Item {
    float *raw;    // [kRawSlots][kRawPlanes][64] floats
    float4 *coef;  // [T+1][2][32]: (Ix, Iy) then (It, -den term) as column pairs
    int lane;
    int lcol;      // first column of this lane's 16-byte chunk (clamped into the row)
    int lc2;       // the lane's own column pair (xa, xa+1), or any in-bounds pair
    bool a_first, a_last, b_last, st_a, st_b;
    int xa, y_start, y_end;
    float alpha2;  // p.alpha2, or the square of the device-resident alpha
};

// Copy one row of the strip (5 planes) into ring slot `slot`, 16-byte chunks through L2
// only (lanes copy chunks other lanes read, so each step brackets the copy and its wait
// with warp barriers).
//   wide: 80 chunks; lane l copies chunks l, l+32 and (lanes 0-15) l+64, i.e. planes u|v,
//         Ix|Iy and It for lanes < 16 | >= 16;
//   else: lanes 0-16 copy chunk `lane` of each of the 5 planes (68 floats per plane row).
template <int T>
__device__ __forceinline__ void issue_row(const Item &it, int slot, int row, const SweepParams &p) {
    using G = Geo<T>;
    row = min(max(row, 0), p.H - 1);
    const size_t off = (size_t)row * p.ld + it.lcol;
    if constexpr (G::wide) {
        const bool lo = it.lane < 16;
        float *base = it.raw + slot * (kRawPlanes * G::rw) + 4 * (it.lane & 15);
        cp_async16(base + (lo ? 0 : 1) * G::rw, (lo ? p.u_in : p.v_in) + off);
        cp_async16(base + (lo ? 2 : 3) * G::rw, (lo ? p.Ix : p.Iy) + off);
        if (lo) cp_async16(base + 4 * G::rw, p.It + off);
    } else {
        if (it.lane < G::rw / 4) {
            float *base = it.raw + slot * (kRawPlanes * G::rw) + 4 * it.lane;
            cp_async16(base + 0 * G::rw, p.u_in + off);
            cp_async16(base + 1 * G::rw, p.v_in + off);
            cp_async16(base + 2 * G::rw, p.Ix + off);
            cp_async16(base + 3 * G::rw, p.Iy + off);
            cp_async16(base + 4 * G::rw, p.It + off);
        }
    }
    cp_async_commit();
}

// One streaming step: row k arrives at stage 0, stage s emits sweep s+1 of row k-s-1.
// HEAD: one of the first 2T-2 steps of a segment that starts T or more rows below the
// image top; stage s only runs from its segment step kk = k - k0 = 2s on (see stream_item).
template <int T, bool FAST, bool XEDGE, bool EDGE, bool DUMP, bool HEAD = false>
__device__ __forceinline__ void stream_step(const SweepParams &p, const Item &it, Win<FAST> (&w)[T][2],
                                            int k, int rslot, int cslot, int kk = 0) {
    // Prefetch row k + kPrefetch into the slot row k-1 used, then wait for row k (never
    // beyond the item's last row: rows past it may belong to tiles that a later pass is
    // already rewriting).  A row's chunks are copied by different lanes than the ones
    // reading them, and cp.async.wait_group covers only the caller's own copies: the
    // warp barrier after it makes every lane's completed copies visible to all lanes,
    // and the one before the prefetch keeps it from overwriting a slot another lane is
    // still reading.
    __syncwarp();
    issue_row<T>(it, (rslot + kPrefetch) & (kRawSlots - 1), min(k + kPrefetch, it.y_end - 1 + T), p);
    cp_async_wait<kPrefetch>();
    __syncwarp();

    // stage 0: unpack row k; pack its coefficients with the negated denominator term
    // (-1/den in the fast form, -den in the exact one: the update then adds a product)
    constexpr int RW = Geo<T>::rw;
    const float *raw = it.raw + rslot * (kRawPlanes * RW) + Geo<T>::sh + 2 * it.lane;
    float2 cu[2] = {lds2(raw), lds2(raw + RW)};  // [plane]: the lane's (u, v) column pairs
    {
        const float2 ix = lds2(raw + 2 * RW), iy = lds2(raw + 3 * RW);
        const float2 t2 = lds2(raw + 4 * RW);
        float2 nd;
        if constexpr (FAST) {
            nd = f2(-rcp_approx(fmaf(iy.x, iy.x, fmaf(ix.x, ix.x, it.alpha2))),
                    -rcp_approx(fmaf(iy.y, iy.y, fmaf(ix.y, ix.y, it.alpha2))));
        } else {
            const float2 d = add2(add2(f2(it.alpha2, it.alpha2), mul2r(ix, ix)), mul2r(iy, iy));
            nd = f2(-d.x, -d.y);
        }
        float4 *cs = it.coef + cslot * 64 + it.lane;
        cs[0] = make_float4(ix.x, ix.y, iy.x, iy.y);
        cs[32] = make_float4(t2.x, t2.y, nd.x, nd.y);
    }
    const float2 we2 = f2(p.we, p.we), wc2 = f2(p.wc, p.wc);

#pragma unroll
    for (int s = 0; s < T; ++s) {
        if (HEAD && kk < 2 * s) break;  // warp-uniform; later stages start later still
        const int n = k - s;  // arriving row (input of sweep s+1)
        float2 ub[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float2 c = cu[q];
            const float fromL = __shfl_up_sync(kFull, c.y, 1);
            const float fromR = __shfl_down_sync(kFull, c.x, 1);
            if constexpr (FAST) {
                // left + right of both columns as scalar adds straight into their pair
                float L = fromL, R0 = c.y, R1 = fromR;
                if constexpr (XEDGE) {
                    L = it.a_first ? c.x : L;
                    R0 = it.a_last ? c.x : R0;
                    R1 = it.b_last ? c.y : R1;
                }
                const float2 h = f2(__fadd_rn(L, R0), __fadd_rn(c.x, R1));
                ub[q] = win_step_h<EDGE>(w[s][q], h, c, n, p.H, we2, wc2);
            } else {
                float2 l = f2(fromL, c.x), r = f2(c.y, fromR);
                if constexpr (XEDGE) {
                    l.x = it.a_first ? c.x : l.x;
                    r.x = it.a_last ? c.x : r.x;
                    r.y = it.b_last ? c.y : r.y;
                }
                ub[q] = win_step<EDGE>(w[s][q], l, c, r, n, p.H, we2, wc2);
            }
        }
        // pointwise update of row n-1 with its coefficients
        int rs = cslot - (s + 1);
        if (rs < 0) rs += Geo<T>::coef_slots;
        const float4 *cr = it.coef + rs * 64 + it.lane;
        const float4 A = cr[0], B = cr[32];
        const float2 cx = f2(A.x, A.y), cy = f2(A.z, A.w), ct = f2(B.x, B.y), nd = f2(B.z, B.w);
        const float2 ubar = ub[0], vbar = ub[1];
        if constexpr (FAST) {
            // -t = (Ix ubar + Iy vbar + It) * (-1/den); u = ubar + Ix (-t) = ubar - Ix t
            const float2 nt = mul2(fma2(cx, ubar, fma2(cy, vbar, ct)), nd);
            cu[0] = fma2(cx, nt, ubar);
            cu[1] = fma2(cy, nt, vbar);
        } else {
            // t = ((Ix ubar + Iy vbar) + It) / den and u = ubar - Ix t, with -t = r / (-den)
            const float2 r = add2(add2(mul2r(cx, ubar), mul2r(cy, vbar)), ct);
            const float2 nt = f2(__fdiv_rn(r.x, nd.x), __fdiv_rn(r.y, nd.y));
            cu[0] = add2(ubar, mul2r(cx, nt));
            cu[1] = add2(vbar, mul2r(cy, nt));
        }
        if constexpr (DUMP) {  // write sweep s+1 of row k-s-1 (state dumps)
            const int rr = k - s - 1;
            if (rr >= it.y_start && rr < it.y_end) {
                const size_t off = (size_t)rr * p.ld + it.xa;
                if (it.st_a && it.st_b) {
                    *reinterpret_cast<float2 *>(p.dump_u[s] + off) = cu[0];
                    *reinterpret_cast<float2 *>(p.dump_v[s] + off) = cu[1];
                } else if (it.st_a) {
                    p.dump_u[s][off] = cu[0].x;
                    p.dump_v[s][off] = cu[1].x;
                }
            }
        }
    }

    // store sweep T of row k - T
    const int r = k - T;
    if (r >= it.y_start && r < it.y_end) {
        const size_t off = (size_t)r * p.ld + it.xa;
        if (it.st_a && it.st_b) {
            *reinterpret_cast<float2 *>(p.u_out + off) = cu[0];
            *reinterpret_cast<float2 *>(p.v_out + off) = cu[1];
        } else if (it.st_a) {
            p.u_out[off] = cu[0].x;
            p.v_out[off] = cu[1].x;
        }
    }
}

// UNR: the main loop body holds two steps; the per-pass kernel runs it rolled from depth 3 up,
// where the shorter code measured faster at every image size (hs_sweep.cu).
template <int T, bool FAST, bool XEDGE, bool DUMP, bool UNR = true>
__device__ __forceinline__ void stream_item(const SweepParams &p, const Item &it) {
    const int k0 = max(0, it.y_start - T);
    const int k_end = it.y_end - 1 + T;
    Win<FAST> w[T][2];
#pragma unroll
    for (int s = 0; s < T; ++s)
#pragma unroll
        for (int q = 0; q < 2; ++q) w[s][q] = Win<FAST>{};

#pragma unroll
    for (int i = 0; i < kPrefetch; ++i) issue_row<T>(it, i, k0 + i, p);

    // Steps in [klo, khi] have no stage at row 0 or past row H-2: no clamp logic.
    const int klo = max(k0, T);
    const int khi = min(k_end, p.H - 2);
    int k = k0, rslot = 0, cslot = 0;
    auto advance = [&]() {
        ++k;
        rslot = (rslot + 1) & (kRawSlots - 1);
        cslot = (cslot + 1 == Geo<T>::coef_slots) ? 0 : cslot + 1;
    };
    // A segment starting T or more rows below the top (k0 = y_start - T > 0) needs stage s's
    // output only from row y_start - (T-1-s) = k0 + s + 1 on, which it first emits at
    // segment step 2s + 2, from the rows it receives at steps 2s and 2s + 1 (stage s-1's
    // first valid rows).  Stage s therefore does nothing useful before step 2s: the first
    // 2T-2 steps skip those stages, T(T-1) stage-steps per segment.  (Their rows lie above
    // y_start, so no dump or store is skipped.)
    if constexpr (!DUMP) {
        if (k0 >= T && k0 + 2 * T - 2 <= khi) {
            for (int kk = 0; kk < 2 * T - 2; ++kk, advance())
                stream_step<T, FAST, XEDGE, false, DUMP, true>(p, it, w, k, rslot, cslot, kk);
        }
    }
    if (klo + 1 <= khi) {
        for (; k < klo; advance()) stream_step<T, FAST, XEDGE, true, DUMP>(p, it, w, k, rslot, cslot);
        if constexpr (UNR) {
            while (k + 1 <= khi) {
                stream_step<T, FAST, XEDGE, false, DUMP>(p, it, w, k, rslot, cslot);
                advance();
                stream_step<T, FAST, XEDGE, false, DUMP>(p, it, w, k, rslot, cslot);
                advance();
            }
        } else {
#pragma unroll 1
            for (; k <= khi; advance()) stream_step<T, FAST, XEDGE, false, DUMP>(p, it, w, k, rslot, cslot);
        }
        // Here k <= H-1, so row H-1 reaches every stage in the tail loop below.  The
        // bottom-clamp values are written and read only there; dropping the head loop's
        // copies keeps them out of the main loop's live registers.
        if constexpr (!FAST) {
#pragma unroll
            for (int s = 0; s < T; ++s)
#pragma unroll
                for (int q = 0; q < 2; ++q) w[s][q].l1 = w[s][q].c1 = w[s][q].r1 = f2(0.f, 0.f);
        }
    }
    for (; k <= k_end; advance()) stream_step<T, FAST, XEDGE, true, DUMP>(p, it, w, k, rslot, cslot);
    cp_async_wait<0>();
}


// ---- host helpers shared by the per-pass and batched launches (hs_sweep.cu)

struct ResolvedConfig {
    int T;
    bool T_default;  // hs_config.sweeps_per_pass was 0: T may follow the image size
    int seg_rows;  // 0 = derive per pass
    bool fast;
    int layout;    // hs_config.layout: 0 automatic, 1 two columns per lane, 2 four
    float we, wc;
};
// whether the sweeps of an H x W image (or a batch averaging that size) run in the
// 4-columns-per-lane layout
bool use_wide(const ResolvedConfig &rc, long pixels);
hs_status resolve_config(const hs_config *cfg, ResolvedConfig *out);
// for the per-pair sweep: when no depth was given, the measured default for an H x W image
void apply_shape_default(ResolvedConfig &rc, int H, int W);
int strip_cols_for(int T);
int default_seg_rows(int H, int nstrips, int T);
hs_status launch_pass(int T, bool fast, const SweepParams &pp, cudaStream_t s);
// `iters` sweeps; the state starts in (u0, v0) for an even number of passes, in (u1, v1)
// for an odd one, and always ends in (u0, v0).  alpha_dev, if set, overrides alpha2.
hs_status run_passes_dev(const float *Ix, const float *Iy, const float *It, int H, int W, int ld,
                         float alpha2, const float *alpha_dev, int iters, float *u0, float *v0,
                         float *u1, float *v1, const ResolvedConfig &rc, cudaStream_t stream);
inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Fill the per-warp context for (strip, seg) of the pass described by p.
template <int T>
__device__ __forceinline__ void init_item(Item &it, const SweepParams &p, int strip, int seg,
                                          int lane, float *wbase) {
    using G = Geo<T>;
    const int x0 = strip * G::strip - G::halo;
    it.raw = wbase;
    it.coef = reinterpret_cast<float4 *>(wbase + G::raw_floats);
    it.lane = lane;
    it.xa = x0 + 2 * lane;
    const int xb = it.xa + 1;
    // the lane's 16-byte chunk: its start and ld are multiples of 4, so a chunk lies wholly
    // inside or outside the row; outside ones copy any in-bounds chunk (their columns never
    // feed a stored pixel)
    const int xc = G::wide ? x0 + 4 * (lane & 15) : x0 - G::sh + 4 * lane;
    it.lcol = (xc >= 0 && xc + 4 <= p.ld) ? xc : 0;
    it.lc2 = (it.xa >= 0 && it.xa < p.W) ? it.xa : 0;  // xa is even and ld % 4 == 0
    it.a_first = (it.xa == 0);
    it.a_last = (it.xa == p.W - 1);
    it.b_last = (xb == p.W - 1);
    const int vlo = strip * G::strip, vhi = min(vlo + G::strip, p.W);
    it.st_a = (it.xa >= vlo && it.xa < vhi);
    it.st_b = (xb >= vlo && xb < vhi);
    it.y_start = seg * p.seg_rows;
    it.y_end = min(p.H, it.y_start + p.seg_rows);
    it.alpha2 = p.alpha_dev ? __fmul_rn(__ldg(p.alpha_dev), __ldg(p.alpha_dev)) : p.alpha2;
}

// Run one work item; only strips reaching an image side need the horizontal clamps.
// DUMP (the training recompute) also writes every stage's sweep to p.dump_u/v; it is a
// template parameter so the plain kernels carry no per-stage branch.
template <int T, bool FAST, bool DUMP = false, bool UNR = true>
__device__ __forceinline__ void run_item(const SweepParams &p, const Item &it) {
    const int x0 = it.xa - 2 * it.lane;
    if (x0 <= 0 || x0 + kWarpCols >= p.W) stream_item<T, FAST, true, DUMP, UNR>(p, it);
    else stream_item<T, FAST, false, DUMP, UNR>(p, it);
}

}  // namespace hs
