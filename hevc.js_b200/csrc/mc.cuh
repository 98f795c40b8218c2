// mc.cuh — motion-compensated prediction (perform_inter_prediction,
// src/decoding/interpolation.cpp:306-411; interpolate_luma :45-127, interpolate_chroma
// :133-209, weighted_pred_default :215-240, weighted_pred_explicit :246-300).
//
// One thread per strip: 4 columns x up to 16 rows of one PU in one plane.  Per reference
// list the thread walks the rows of its reference window once, two rows at a time:
//   1. the two rows are read as aligned 32-bit words (the next two rows' loads are issued
//      before these are used, so a row's latency overlaps the previous rows' arithmetic);
//   2. each row is realigned with funnel shifts and filtered horizontally with dp4a
//      (signed 8-bit taps x unsigned samples), and the two rows' results are packed per
//      column into one word of int16 pairs (row 2m low, row 2m+1 high);
//   3. once the window holds NT/2 + 1 such pair words per column, the vertical filter
//      produces output rows 2m and 2m + 1 with dp2a (two int16 intermediates x two 8-bit
//      taps per instruction: NT/2 for the even row, NT/2 + 1 for the odd row);
//   4. the outputs are weighted (default or explicit, one formula with per-plane
//      constants), saturated and packed to bytes with cvt.pack.sat, and stored as words.
// A bi-predicted strip keeps its list-0 predictions in shared memory (int16 x 4 per row)
// until the list-1 pass combines them.
//
// Every fractional phase goes through this one 2-D path.  With the phase-0 taps
// (0,0,0,64,0,0,0,0 / 0,64,0,0) it reproduces the reference's special cases exactly at
// 8 bits: horizontal-only gives (64 * h) >> 6 = h, vertical-only gives (sum 64 * v * s) >> 6,
// full-pel gives 64 * 64 * s >> 6 = s << 6, and no intermediate leaves int16
// (|horizontal| <= 255 * 88 and |vertical| <= 30855 for 8-bit samples), so the reference's
// int16 casts never wrap.  Samples outside the picture repeat the edge (refClamp, :64-68).
//
// The host orders the strips of a launch by (bi-predicted first, window inside the picture
// first, taller first), so the threads of a warp take the same path for the same number of
// rows; inside a class strips stay in PU order, so neighbouring threads read neighbouring
// words.
#pragma once

#include "device_common.cuh"

namespace hevcgpu {

__host__ __device__ constexpr uint32_t pack4(int a, int b, int c, int d) {
    return (uint32_t)(uint8_t)a | ((uint32_t)(uint8_t)b << 8) | ((uint32_t)(uint8_t)c << 16) |
           ((uint32_t)(uint8_t)d << 24);
}

// luma_filter / chroma_filter (interpolation.cpp:17-38); byte i weighs sample offset i-3
// (luma) or i-1 (chroma)
__constant__ uint32_t c_luma_pk[4][2] = {{pack4(0, 0, 0, 64), pack4(0, 0, 0, 0)},
                                         {pack4(-1, 4, -10, 58), pack4(17, -5, 1, 0)},
                                         {pack4(-1, 4, -11, 40), pack4(40, -11, 4, -1)},
                                         {pack4(0, 1, -5, 17), pack4(58, -10, 4, -1)}};
__constant__ uint32_t c_chroma_pk[8] = {pack4(0, 64, 0, 0),   pack4(-2, 58, 10, -2), pack4(-4, 54, 16, -2),
                                        pack4(-6, 46, 28, -4), pack4(-4, 36, 36, -4), pack4(-4, 28, 46, -6),
                                        pack4(-2, 16, 54, -4), pack4(-2, 10, 58, -2)};

__device__ __forceinline__ int dp4a_su(uint32_t taps, uint32_t samples, int c) {
    int d;
    asm("dp4a.s32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(taps), "r"(samples), "r"(c));
    return d;
}
// c + a.lo16 * b.byte0 + a.hi16 * b.byte1 (lo) or bytes 2, 3 (hi), all signed
__device__ __forceinline__ int dp2a_lo(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp2a.lo.s32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ int dp2a_hi(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp2a.hi.s32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
// v0..v3 saturated to 0..255 and packed as bytes 0..3 (PTX cvt.pack.sat: the low 16 bits
// of c move up by 16 and a, b take bits 15..8 and 7..0).
__device__ __forceinline__ uint32_t pack_sat_u8x4(int v0, int v1, int v2, int v3) {
    uint32_t t, d;
    asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, 0;" : "=r"(t) : "r"(v3), "r"(v2));
    asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(v1), "r"(v0), "r"(t));
    return d;
}

// Strip work item, 32 bits: PU index (bits 0-19), strip column / 4 (20-23), strip row / 16
// (24-25), rows code (26-28: luma rows / 4 - 1, chroma rows / 2 - 1), chroma plane (29:
// 0 Cb, 1 Cr).  Offsets and rows are in samples of the strip's plane.
constexpr int MC_THREADS = 128;
#ifndef HEVCGPU_MC_MIN_CTAS
#define HEVCGPU_MC_MIN_CTAS 6   // CTAs per SM the register budget is sized for (80 registers)
#endif
constexpr int MC_STRIP_ROWS = 16;
constexpr int MC_MAX_PUS = 1 << 20;
__host__ __device__ constexpr uint32_t mc_item(int pu, int sx, int sy, int rows, bool chroma, int plane) {
    return (uint32_t)pu | ((uint32_t)(sx >> 2) << 20) | ((uint32_t)(sy >> 4) << 24) |
           ((uint32_t)(chroma ? (rows >> 1) - 1 : (rows >> 2) - 1) << 26) | ((uint32_t)plane << 29);
}

// Per-plane geometry of a strip.
template <bool CHROMA>
struct McGeom {
    static constexpr int NT = CHROMA ? 4 : 8;      // taps
    static constexpr int HALF = NT / 2 - 1;        // window starts HALF samples left / above
    static constexpr int SUB = CHROMA ? 2 : 1;
    static constexpr int NW = CHROMA ? 3 : 4;      // aligned words per window row
    static constexpr int NP = NT / 2 + 1;          // pair words per column in the vertical window
    static constexpr int MAXP = MC_STRIP_ROWS / 2 + NT / 2;   // row pairs of the tallest strip
};

// True when every word a strip reads for one list lies inside the picture: window rows
// y0 .. y0 + rows + NT - 1 (one row beyond the NT - 1 the filter needs, read for the
// zero tap of the last odd output row) and bytes x0 .. x0 + NT + 2, from the aligned word
// at x0 & ~3 (NW words, inside the row pitch).  Shared with the host, which sorts strips
// by it.
template <bool CHROMA>
__host__ __device__ __forceinline__ bool mc_inside(int x0, int y0, int rows, int pw, int ph, int pitch) {
    using G_ = McGeom<CHROMA>;
    return x0 >= 0 && y0 >= 0 && x0 + G_::NT + 3 <= pw && (x0 & ~3) + 4 * G_::NW <= pitch &&
           y0 + rows + G_::NT <= ph;
}

// Weighting of one plane (weighted_pred_default / weighted_pred_explicit) as one form:
// uni: ((p * w0 + add) >> shift) + o;  bi: (p0 * w0 + p1 * w1 + add) >> shift.
struct McWeights {
    int w0, w1, add, shift, o;
};
__device__ __forceinline__ McWeights mc_weights(const hevc_wp_t* wp, bool bi, bool use0, int ci) {
    McWeights r;
    if (!wp) {
        r.w0 = 1;
        r.w1 = 1;
        r.add = bi ? 64 : 32;
        r.shift = bi ? 7 : 6;
        r.o = 0;
        return r;
    }
    const int lw = wp->log2wd[ci ? 1 : 0];
    if (bi) {
        r.w0 = wp->w[0][ci];
        r.w1 = wp->w[1][ci];
        r.add = (wp->o[0][ci] + wp->o[1][ci] + 1) << lw;
        r.shift = lw + 1;
        r.o = 0;
    } else {
        const int l = use0 ? 0 : 1;
        r.w0 = wp->w[l][ci];
        r.w1 = 0;
        r.add = 1 << (lw - 1);
        r.shift = lw;
        r.o = wp->o[l][ci];
    }
    return r;
}

// NW aligned words of window row y from byte xa (a multiple of 4) onwards.  INSIDE: the
// whole window lies inside the picture and the row is read at rowp.  Otherwise the
// samples are edge-clamped (refClamp): the row index is clamped, and since a plane's
// width is a multiple of 4 (pictures are multiples of 8), an aligned word lies either
// wholly inside the row or wholly left or right of it; a word left of the row is the
// row's first sample four times, a word right of it the row's last sample four times.
template <int NW, bool INSIDE>
__device__ __forceinline__ void mc_row(const uint8_t* rowp, const uint8_t* plane, int pitch, int pw, int ph, int y,
                                       int xa, uint32_t (&w)[NW]) {
    if constexpr (INSIDE) {
        const uint32_t* p = reinterpret_cast<const uint32_t*>(rowp);
#pragma unroll
        for (int q = 0; q < NW; q++) w[q] = __ldg(p + q);
    } else {
        const uint8_t* row = plane + (int64_t)clip3(0, ph - 1, y) * pitch;
#pragma unroll
        for (int q = 0; q < NW; q++) {
            const int a = xa + 4 * q;
            const uint32_t v = __ldg(reinterpret_cast<const uint32_t*>(row + clip3(0, pw - 4, a)));
            w[q] = a < 0 ? __byte_perm(v, 0, 0x0000) : (a > pw - 4 ? __byte_perm(v, 0, 0x3333) : v);
        }
    }
}

// Horizontal filter of one window row (words w realigned by sh bits) into h[0..3].
template <bool CHROMA>
__device__ __forceinline__ void mc_hrow(const uint32_t (&w)[McGeom<CHROMA>::NW], int sh, uint32_t tlo, uint32_t thi,
                                        int (&h)[4]) {
    const uint32_t s0 = __funnelshift_r(w[0], w[1], sh), s1 = __funnelshift_r(w[1], w[2], sh);
    if constexpr (CHROMA) {
#pragma unroll
        for (int j = 0; j < 4; j++) h[j] = dp4a_su(tlo, __funnelshift_r(s0, s1, 8 * j), 0);
    } else {
        const uint32_t s2 = __funnelshift_r(w[2], w[3], sh);
#pragma unroll
        for (int j = 0; j < 4; j++)
            h[j] = dp4a_su(thi, __funnelshift_r(s1, s2, 8 * j), dp4a_su(tlo, __funnelshift_r(s0, s1, 8 * j), 0));
    }
}

// One list of one strip: prediction (before weighting, at 14-bit scale) of 4 columns x
// `rows` rows whose window starts at (x0, y0) with phases (fx, fy) of the plane; emit(k, p)
// receives output rows k = 0, 1, 2, ... in order.  INSIDE: the window lies inside the
// picture (mc_inside), so rows are read straight; else every row and byte is clamped.
template <bool CHROMA, bool INSIDE, typename Emit>
__device__ __forceinline__ void mc_list(const uint8_t* plane, int pitch, int pw, int ph, int x0, int y0, int fx, int fy,
                                        int rows, Emit&& emit) {
    using G_ = McGeom<CHROMA>;
    constexpr int NT = G_::NT, NW = G_::NW, NP = G_::NP;
    const int xa = x0 & ~3, sh = 8 * (x0 & 3);
    uint32_t tlo, thi = 0, e0, e1 = 0, o0, o1, o2 = 0;   // horizontal taps; vertical tap words
    if constexpr (CHROMA) {
        tlo = c_chroma_pk[fx];
        const uint32_t v = c_chroma_pk[fy];
        e0 = v;
        o0 = v << 8;
        o1 = v >> 24;
    } else {
        tlo = c_luma_pk[fx][0];
        thi = c_luma_pk[fx][1];
        const uint32_t v0 = c_luma_pk[fy][0], v1 = c_luma_pk[fy][1];
        e0 = v0;
        e1 = v1;
        o0 = v0 << 8;
        o1 = __funnelshift_l(v0, v1, 8);
        o2 = v1 >> 24;
    }
    const int np = rows / 2 + NT / 2;   // window row pairs
    const uint8_t* rowp = plane + (int64_t)y0 * pitch + xa;
    uint32_t nxt[2][NW];
    uint32_t win[NP][4];
#pragma unroll
    for (int r = 0; r < 2; r++)
        mc_row<NW, INSIDE>(rowp + (int64_t)r * pitch, plane, pitch, pw, ph, y0 + r, xa, nxt[r]);
#pragma unroll
    for (int p = 0; p < G_::MAXP; p++) {
        if (p >= np) break;
        uint32_t cur[2][NW];
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
            for (int q = 0; q < NW; q++) cur[r][q] = nxt[r][q];
        if (p + 1 < np) {
            rowp += 2 * (int64_t)pitch;
#pragma unroll
            for (int r = 0; r < 2; r++)
                mc_row<NW, INSIDE>(rowp + (int64_t)r * pitch, plane, pitch, pw, ph, y0 + 2 * p + 2 + r, xa, nxt[r]);
        }
        int ha[4], hb[4];
        mc_hrow<CHROMA>(cur[0], sh, tlo, thi, ha);
        mc_hrow<CHROMA>(cur[1], sh, tlo, thi, hb);
#pragma unroll
        for (int c = 0; c < 4; c++) win[p % NP][c] = __byte_perm((uint32_t)ha[c], (uint32_t)hb[c], 0x5410);
        if (p >= NT / 2) {
            const int m = p - NT / 2;
            int pe[4], po[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const uint32_t w0 = win[m % NP][c], w1 = win[(m + 1) % NP][c], w2 = win[(m + 2) % NP][c];
                if constexpr (CHROMA) {
                    pe[c] = dp2a_hi(w1, e0, dp2a_lo(w0, e0, 0)) >> 6;
                    po[c] = dp2a_lo(w2, o1, dp2a_hi(w1, o0, dp2a_lo(w0, o0, 0))) >> 6;
                } else {
                    const uint32_t w3 = win[(m + 3) % NP][c], w4 = win[(m + 4) % NP][c];
                    pe[c] = dp2a_hi(w3, e1, dp2a_lo(w2, e1, dp2a_hi(w1, e0, dp2a_lo(w0, e0, 0)))) >> 6;
                    po[c] = dp2a_lo(w4, o2, dp2a_hi(w3, o1, dp2a_lo(w2, o1, dp2a_hi(w1, o0, dp2a_lo(w0, o0, 0))))) >> 6;
                }
            }
            emit(2 * m, pe);
            emit(2 * m + 1, po);
        }
    }
}

// Luma strips and chroma strips are separate launches (separate item lists).
template <bool CHROMA>
__global__ void __launch_bounds__(MC_THREADS, HEVCGPU_MC_MIN_CTAS) k_mc(const __grid_constant__ SegTable st) {
    using G_ = McGeom<CHROMA>;
    constexpr int SUB = G_::SUB;
    __shared__ uint2 s_pred[MC_STRIP_ROWS][MC_THREADS];   // list-0 predictions of bi strips
    const int tid = threadIdx.x;
    const Seg& sg = st.s[find_seg(st, blockIdx.x)];
    const int item = (blockIdx.x - sg.block0) * MC_THREADS + tid;
    if (item >= sg.n_items) return;
    const uint32_t it = static_cast<const uint32_t*>(sg.items)[item];
    const PicDesc& P = *sg.pic;
    const hevc_pu_t pu = P.pus[it & (MC_MAX_PUS - 1)];
    const int sx = (int)((it >> 20) & 15) << 2, sy = (int)((it >> 24) & 3) << 4;
    const int rows = CHROMA ? 2 * (int)(((it >> 26) & 7) + 1) : 4 * (int)(((it >> 26) & 7) + 1);
    const int ci = CHROMA ? 1 + (int)((it >> 29) & 1) : 0;
    const bool use0 = pu.ref_idx[0] >= 0, use1 = pu.ref_idx[1] >= 0, bi = use0 && use1;
    const int pw = P.width / SUB, ph = P.height / SUB, pitch = CHROMA ? P.pitch_c : P.pitch_y;
    const int64_t poff = ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr);
    const int x = pu.x / SUB + sx, y = pu.y / SUB + sy;
    const bool wide = !CHROMA || pu.w / SUB - sx >= 4;   // chroma strips of 2-wide PU parts store 2 columns
    const McWeights wt = mc_weights(pu.wp >= 0 ? &P.wp[pu.wp] : nullptr, bi, use0, ci);
    uint8_t* const out = P.rec + poff + (int64_t)y * pitch + x;
    const int wlast = bi ? wt.w1 : wt.w0;   // weight of the last pass's list
    if constexpr (!CHROMA) {
        // the strip's 4x4 units of the motion grid (the Bs derivation's PU motion), as the
        // three words of a MotionEnt: mv[0], mv[1], ref_idx[0..1] (padding zero)
        if (P.mot) {
            const uint32_t m0 = (uint32_t)(uint16_t)pu.mv[0][0] | ((uint32_t)(uint16_t)pu.mv[0][1] << 16);
            const uint32_t m1 = (uint32_t)(uint16_t)pu.mv[1][0] | ((uint32_t)(uint16_t)pu.mv[1][1] << 16);
            const uint32_t m2 = (uint32_t)(uint8_t)pu.ref_idx[0] | ((uint32_t)(uint8_t)pu.ref_idx[1] << 8);
            const int gw = P.width / 4;
            uint32_t* g = reinterpret_cast<uint32_t*>(P.mot + (int64_t)(y >> 2) * gw + (x >> 2));
            for (int k = 0; k < rows / 4; k++, g += 3 * gw) {
                g[0] = m0;
                g[1] = m1;
                g[2] = m2;
            }
        }
    }

#pragma unroll 1
    for (int q = 0; q < (bi ? 2 : 1); q++) {
        const int l = bi ? q : (use0 ? 0 : 1);
        // list selection by value (no runtime index into the PU record, which would put it
        // in local memory)
        const int mvx = l ? pu.mv[1][0] : pu.mv[0][0], mvy = l ? pu.mv[1][1] : pu.mv[0][1];
        const uint8_t* ref = (l ? P.ref[1][pu.ref_idx[1]] : P.ref[0][pu.ref_idx[0]]) + poff;
        const int x0 = x + (CHROMA ? (mvx >> 3) : (mvx >> 2)) - G_::HALF;
        const int y0 = y + (CHROMA ? (mvy >> 3) : (mvy >> 2)) - G_::HALF;
        const int fx = CHROMA ? (mvx & 7) : (mvx & 3), fy = CHROMA ? (mvy & 7) : (mvy & 3);
        const bool stash = bi && q == 0;
        uint8_t* orow = out;   // output row k, advanced by one row per emitted row
        auto emit = [&](int k, const int (&p)[4]) {
            if (stash) {
                s_pred[k][tid] = make_uint2(__byte_perm((uint32_t)p[0], (uint32_t)p[1], 0x5410),
                                            __byte_perm((uint32_t)p[2], (uint32_t)p[3], 0x5410));
                return;
            }
            int v[4];
#pragma unroll
            for (int c = 0; c < 4; c++) v[c] = p[c] * wlast + wt.add;
            if (bi) {
                const uint2 s = s_pred[k][tid];
                v[0] += (int)(int16_t)(s.x & 0xFFFF) * wt.w0;
                v[1] += ((int)s.x >> 16) * wt.w0;
                v[2] += (int)(int16_t)(s.y & 0xFFFF) * wt.w0;
                v[3] += ((int)s.y >> 16) * wt.w0;
            }
#pragma unroll
            for (int c = 0; c < 4; c++) v[c] = (v[c] >> wt.shift) + wt.o;
            const uint32_t b = pack_sat_u8x4(v[0], v[1], v[2], v[3]);
            uint8_t* const o = orow;
            orow += pitch;
            if (!CHROMA || (wide && !(x & 3))) {
                *reinterpret_cast<uint32_t*>(o) = b;   // luma strips are 4 wide and 4-aligned
            } else {
                *reinterpret_cast<uint16_t*>(o) = (uint16_t)b;
                if (wide) *reinterpret_cast<uint16_t*>(o + 2) = (uint16_t)(b >> 16);
            }
        };
        if (mc_inside<CHROMA>(x0, y0, rows, pw, ph, pitch))
            mc_list<CHROMA, true>(ref, pitch, pw, ph, x0, y0, fx, fy, rows, emit);
        else
            mc_list<CHROMA, false>(ref, pitch, pw, ph, x0, y0, fx, fy, rows, emit);
    }
}

}  // namespace hevcgpu
