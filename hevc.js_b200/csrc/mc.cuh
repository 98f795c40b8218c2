// mc.cuh — motion-compensated prediction (perform_inter_prediction,
// src/decoding/interpolation.cpp:306-411; interpolate_luma :45-127, interpolate_chroma
// :133-209, weighted_pred_default :215-240, weighted_pred_explicit :246-300).
//
// One warp per block of a PU: up to 16 x 16 luma samples, or up to 8 x 8 samples of both
// chroma planes (lanes 0-15 Cb, 16-31 Cr).  The lanes of a plane
//   1. load the reference windows of the block's lists ((w+7) x (h+7) luma, (w+3) x (h+3)
//      chroma) into shared memory as aligned words, every load of both lists issued before
//      any is used (edge-clamped byte loads where the window leaves the picture: refClamp,
//      :64-68);
//   2. filter each window horizontally with dp4a (signed 8-bit taps x unsigned samples)
//      into int16 intermediates stored as row pairs (I[2m][j], I[2m+1][j]);
//   3. filter vertically with dp2a (two int16 intermediates x two 8-bit taps per
//      instruction), each lane owning one column and an even run of rows so that its pair
//      words and tap words are fixed at compile time;
//   4. weight (default or explicit, one formula with per-plane constants) and store.
//
// Every fractional phase goes through this one 2-D path.  With the phase-0 taps
// (0,0,0,64,0,0,0,0 / 0,64,0,0) it reproduces the reference's special cases exactly at
// 8 bits: horizontal-only gives (64 * h) >> 6 = h, vertical-only gives (sum 64 * v * s) >> 6,
// full-pel gives 64 * 64 * s >> 6 = s << 6, and no intermediate leaves int16
// (|horizontal| <= 255 * 88 and |vertical| <= 30855 for 8-bit samples), so the reference's
// int16 casts never wrap.
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
// log2 of the smallest power of two >= v, for v in 1..16
__device__ __forceinline__ int log2_ceil16(int v) { return v <= 1 ? 0 : (v <= 2 ? 1 : (v <= 4 ? 2 : (v <= 8 ? 3 : 4))); }

// Block work item: a block of one PU in one component (luma, or Cb and Cr together).
struct McBlock {
    int32_t pu;
    uint8_t bx, by;   // block offset inside the PU, in samples of its component
    uint8_t bw, bh;   // luma: up to 16 x 16; chroma: up to 8 x 8
};
constexpr int MC_WARPS = 4;
constexpr int MC_BLOCK_LUMA = 16, MC_BLOCK_CHROMA = 8;

// Per-plane geometry of the warp-cooperative block filter.  The row pitches keep the lanes
// of one shared-memory access in distinct banks for the lane mappings below.
template <bool CHROMA>
struct McGeom {
    static constexpr int NT = CHROMA ? 4 : 8;          // taps
    static constexpr int HALF = NT / 2 - 1;            // window starts HALF samples left / above
    static constexpr int SUB = CHROMA ? 2 : 1;
    static constexpr int LANES = CHROMA ? 16 : 32;     // lanes per plane
    static constexpr int LLANES = CHROMA ? 4 : 5;      // log2(LANES)
    static constexpr int ROWS = CHROMA ? 12 : 24;      // window rows (even, >= block + NT - 1)
    static constexpr int WSLOTS = CHROMA ? 4 : 8;      // aligned words per window row, at most
    static constexpr int WPITCH = CHROMA ? 6 : 10;     // window row pitch (words)
    static constexpr int PPITCH = CHROMA ? 12 : 20;    // pair row pitch (words)
    static constexpr int PROWS = CHROMA ? 8 : 16;      // pair rows
    static constexpr int R = CHROMA ? 4 : 8;           // output rows a lane owns, at most (even)
    static constexpr int NPW = (R + NT) / 2;           // pair words a lane reads
    static constexpr int LOADS = ROWS * WSLOTS / LANES;
    static constexpr int PLANES = CHROMA ? 2 : 1;
    // words per plane, padded to an odd multiple of 16 so the two chroma planes start 16
    // banks apart
    static constexpr int PLANE_WORDS = ((2 * ROWS * WPITCH + PROWS * PPITCH + 31) / 32) * 32 + 16;
    static constexpr int WARP_WORDS = PLANES * PLANE_WORDS;
};

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

// One block of plane ci by the plane's lanes (hl = lane within the plane), with the
// plane's shared memory smem ([2][ROWS][WPITCH] windows, then [PROWS][PPITCH] pairs).
template <bool CHROMA>
__device__ __forceinline__ void mc_block(const PicDesc& P, const hevc_pu_t& pu, const McBlock& b, uint32_t* smem,
                                         int hl, int ci) {
    using G_ = McGeom<CHROMA>;
    constexpr int NT = G_::NT, HALF = G_::HALF, SUB = G_::SUB, LANES = G_::LANES, R = G_::R, NPW = G_::NPW;
    uint32_t* s_ref = smem;
    uint32_t* s_pairs = smem + 2 * G_::ROWS * G_::WPITCH;
    const bool use0 = pu.ref_idx[0] >= 0, use1 = pu.ref_idx[1] >= 0, bi = use0 && use1;
    const int nl = bi ? 2 : 1;
    const int pw = P.width / SUB, ph = P.height / SUB, pitch = CHROMA ? P.pitch_c : P.pitch_y;
    const int64_t poff = ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr);
    const int x = pu.x / SUB + b.bx, y = pu.y / SUB + b.by, bw = b.bw, bh = b.bh;
    const int W = bw + NT - 1, H = bh + NT - 1;
    const uint8_t* ref0 = use0 ? P.ref[0][pu.ref_idx[0]] + poff : nullptr;
    const uint8_t* ref1 = use1 ? P.ref[1][pu.ref_idx[1]] + poff : nullptr;
    uint8_t* const rec = P.rec + poff;
    const McWeights wt = mc_weights(pu.wp >= 0 ? &P.wp[pu.wp] : nullptr, bi, use0, ci);

    // 1. reference windows of every list, all loads before any store
    int sh0 = 0, sh1 = 0, fx0 = 0, fx1 = 0, fy0 = 0, fy1 = 0;   // per list, as scalars
#pragma unroll
    for (int q = 0; q < 2; q++) {
        if (q >= nl) break;
        const int l = bi ? q : (use0 ? 0 : 1);
        const int mvx = l ? pu.mv[1][0] : pu.mv[0][0], mvy = l ? pu.mv[1][1] : pu.mv[0][1];
        const int xi = x + (CHROMA ? (mvx >> 3) : (mvx >> 2)), yi = y + (CHROMA ? (mvy >> 3) : (mvy >> 2));
        const int fx = CHROMA ? (mvx & 7) : (mvx & 3), fy = CHROMA ? (mvy & 7) : (mvy & 3);
        const int x0 = xi - HALF, y0 = yi - HALF, xa = x0 & ~3, nw = ((x0 - xa) + W + 3) >> 2;
        (q ? fx1 : fx0) = fx;
        (q ? fy1 : fy0) = fy;
        (q ? sh1 : sh0) = 8 * (x0 - xa);
        const uint8_t* plane = l ? ref1 : ref0;
        const bool fast = x0 >= 0 && y0 >= 0 && xa + 4 * nw <= pw && y0 + H <= ph;
        uint32_t v[G_::LOADS];
#pragma unroll
        for (int k = 0; k < G_::LOADS; k++) {
            const int idx = hl + LANES * k, r = idx / G_::WSLOTS, w = idx % G_::WSLOTS;
            v[k] = 0;
            if (r >= H || w >= nw) continue;
            if (fast) {
                v[k] = __ldg(reinterpret_cast<const uint32_t*>(plane + (int64_t)(y0 + r) * pitch + xa) + w);
            } else {
                const uint8_t* row = plane + (int64_t)clip3(0, ph - 1, y0 + r) * pitch;
#pragma unroll
                for (int t = 0; t < 4; t++)
                    v[k] |= (uint32_t)__ldg(row + clip3(0, pw - 1, xa + 4 * w + t)) << (8 * t);
            }
        }
#pragma unroll
        for (int k = 0; k < G_::LOADS; k++) {
            const int idx = hl + LANES * k, r = idx / G_::WSLOTS, w = idx % G_::WSLOTS;
            if (r < H && w < nw) s_ref[(q * G_::ROWS + r) * G_::WPITCH + w] = v[k];
        }
    }
    __syncwarp();

    // vertical-pass mapping: lane -> column j (of bw rounded up to a power of two) and the
    // rows [k0, k0 + rr), rr even; shifts and masks only
    const int lbw = log2_ceil16(bw), lgrp = G_::LLANES - lbw;
    const int rr = ((bh + (2 << lgrp) - 1) >> (lgrp + 1)) << 1;
    const int j = hl & ((1 << lbw) - 1), grp = hl >> lbw, k0 = grp * rr;
    const bool vlane = j < bw && k0 < bh;
    int pred0[R];
    uint8_t* out = rec + (int64_t)(y + k0) * pitch + x + j;
    // horizontal-pass tasks: (row pair m, 4-column group g), groups rounded up to a power of two
    const int lg = log2_ceil16((bw + 3) >> 2), G = (bw + 3) >> 2, npairs = (H + 1) >> 1;

#pragma unroll 1
    for (int q = 0; q < nl; q++) {
        // 2. horizontal pass
        const int sh = q ? sh1 : sh0, fxq = q ? fx1 : fx0, fyq = q ? fy1 : fy0;
        uint32_t tlo, thi = 0;
        if constexpr (CHROMA) {
            tlo = c_chroma_pk[fxq];
        } else {
            tlo = c_luma_pk[fxq][0];
            thi = c_luma_pk[fxq][1];
        }
        for (int t = hl; t < (npairs << lg); t += LANES) {
            const int m = t >> lg, g = t & ((1 << lg) - 1);
            if (g >= G) continue;
            int iv[2][4];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t* row = s_ref + (q * G_::ROWS + 2 * m + h) * G_::WPITCH + g;
                const uint32_t w0 = row[0], w1 = row[1], w2 = row[2];
                const uint32_t s0 = __funnelshift_r(w0, w1, sh), s1 = __funnelshift_r(w1, w2, sh);
                if constexpr (CHROMA) {
#pragma unroll
                    for (int c = 0; c < 4; c++) iv[h][c] = dp4a_su(tlo, __funnelshift_r(s0, s1, 8 * c), 0);
                } else {
                    const uint32_t s2 = __funnelshift_r(w2, row[3], sh);
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        iv[h][c] = dp4a_su(thi, __funnelshift_r(s1, s2, 8 * c),
                                           dp4a_su(tlo, __funnelshift_r(s0, s1, 8 * c), 0));
                }
            }
            uint32_t* dst = s_pairs + m * G_::PPITCH + 4 * g;
#pragma unroll
            for (int c = 0; c < 4; c++) dst[c] = (uint32_t)(iv[0][c] & 0xFFFF) | ((uint32_t)iv[1][c] << 16);
        }
        __syncwarp();

        // 3. vertical pass, 4. weighting and store
        if (vlane) {
            uint32_t e0, e1 = 0, o0, o1, o2 = 0;   // tap words for even and odd output rows
            if constexpr (CHROMA) {
                const uint32_t v = c_chroma_pk[fyq];
                e0 = v;
                o0 = v << 8;
                o1 = v >> 24;
            } else {
                const uint32_t v0 = c_luma_pk[fyq][0], v1 = c_luma_pk[fyq][1];
                e0 = v0;
                e1 = v1;
                o0 = v0 << 8;
                o1 = __funnelshift_l(v0, v1, 8);
                o2 = v1 >> 24;
            }
            uint32_t pwd[NPW];
#pragma unroll
            for (int i = 0; i < NPW; i++) pwd[i] = s_pairs[((k0 >> 1) + i) * G_::PPITCH + j];
#pragma unroll
            for (int i = 0; i < R; i++) {
                if (i >= rr || k0 + i >= bh) break;
                const int m = i >> 1;
                int acc;
                if constexpr (CHROMA) {
                    acc = (i & 1) ? dp2a_lo(pwd[m + 2], o1, dp2a_hi(pwd[m + 1], o0, dp2a_lo(pwd[m], o0, 0)))
                                  : dp2a_hi(pwd[m + 1], e0, dp2a_lo(pwd[m], e0, 0));
                } else {
                    acc = (i & 1) ? dp2a_lo(pwd[m + 4], o2,
                                            dp2a_hi(pwd[m + 3], o1,
                                                    dp2a_lo(pwd[m + 2], o1,
                                                            dp2a_hi(pwd[m + 1], o0, dp2a_lo(pwd[m], o0, 0)))))
                                  : dp2a_hi(pwd[m + 3], e1,
                                            dp2a_lo(pwd[m + 2], e1, dp2a_hi(pwd[m + 1], e0, dp2a_lo(pwd[m], e0, 0))));
                }
                const int p = acc >> 6;
                if (bi) {
                    if (q == 0) pred0[i] = p;
                    else out[(int64_t)i * pitch] = (uint8_t)clip_u8((pred0[i] * wt.w0 + p * wt.w1 + wt.add) >> wt.shift);
                } else {
                    out[(int64_t)i * pitch] = (uint8_t)clip_u8(((p * wt.w0 + wt.add) >> wt.shift) + wt.o);
                }
            }
        }
        __syncwarp();
    }
}

// Luma blocks and chroma blocks are separate launches (separate item lists); one warp per
// block, MC_WARPS blocks per CTA.
template <bool CHROMA>
__global__ void __launch_bounds__(MC_WARPS * 32) k_mc(const __grid_constant__ SegTable st) {
    using G_ = McGeom<CHROMA>;
    __shared__ uint32_t s_mc[MC_WARPS * G_::WARP_WORDS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Seg& sg = st.s[find_seg(st, blockIdx.x)];
    const int item = (blockIdx.x - sg.block0) * MC_WARPS + warp;
    if (item >= sg.n_items) return;
    const McBlock b = static_cast<const McBlock*>(sg.items)[item];
    const PicDesc& P = *sg.pic;
    const hevc_pu_t pu = P.pus[b.pu];
    const int plane = CHROMA ? (lane >> 4) : 0;
    mc_block<CHROMA>(P, pu, b, s_mc + warp * G_::WARP_WORDS + plane * G_::PLANE_WORDS,
                     CHROMA ? (lane & 15) : lane, CHROMA ? 1 + plane : 0);
}

}  // namespace hevcgpu
