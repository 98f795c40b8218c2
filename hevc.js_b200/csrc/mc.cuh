// mc.cuh — motion-compensated prediction (perform_inter_prediction,
// src/decoding/interpolation.cpp:306-411; interpolate_luma :45-127, interpolate_chroma
// :133-209, weighted_pred_default :215-240, weighted_pred_explicit :246-300).
//
// One thread per output strip: 4 columns x up to 16 rows of one PU and one component
// (luma, or Cb and Cr together).  Per reference list the thread walks the rows of its
// reference window once: every window row is read as aligned 32-bit words, realigned with
// funnel shifts, and filtered horizontally with dp4a (signed 8-bit taps x unsigned
// samples); the last 8 (luma) or 4 (chroma) horizontal results live in a rotating register
// window from which the vertical filter produces one output row per window row.
//
// Every fractional phase goes through this one 2-D path.  With the phase-0 taps
// (0,0,0,64,0,0,0,0 / 0,64,0,0) it reproduces the reference's special cases exactly at
// 8 bits: horizontal-only gives (64 * h) >> 6 = h, vertical-only gives (sum 64 * v * s) >> 6,
// full-pel gives 64 * 64 * s >> 6 = s << 6, and no intermediate leaves int16
// (|horizontal| <= 255 * 88 and |vertical| <= 30855 for 8-bit samples), so the reference's
// int16 casts never wrap.  Samples outside the picture repeat the edge (refClamp, :64-68).
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
__device__ __forceinline__ int tap_of(uint32_t pk, int i) { return (int)(int8_t)(pk >> (8 * i)); }

// Strip work item.
struct McStrip {
    int32_t pu;
    uint8_t sx, sy;   // strip offset inside the PU, in samples of its component
    uint8_t h;        // rows (1..16)
    uint8_t pad;
};
constexpr int MC_THREADS = 128;

// NW aligned words of row y covering byte offset xa (multiple of 4) onwards; outside the
// picture the words are assembled from edge-clamped bytes.
template <int NW>
__device__ __forceinline__ void row_words(const uint8_t* plane, int pitch, int pw, int ph, int y, int xa, bool fast,
                                          uint32_t (&w)[NW]) {
    if (fast) {
        const uint32_t* p = reinterpret_cast<const uint32_t*>(plane + (int64_t)y * pitch + xa);
#pragma unroll
        for (int q = 0; q < NW; q++) w[q] = __ldg(p + q);
    } else {
        const uint8_t* row = plane + (int64_t)clip3(0, ph - 1, y) * pitch;
#pragma unroll
        for (int q = 0; q < NW; q++) {
            uint32_t v = 0;
#pragma unroll 1
            for (int b = 0; b < 4; b++) v |= (uint32_t)__ldg(row + clip3(0, pw - 1, xa + 4 * q + b)) << (8 * b);
            w[q] = v;
        }
    }
}

// Final sample of one prediction (weighted_pred_default / weighted_pred_explicit).
__device__ __forceinline__ int weigh(int p0, int p1, bool u0, bool u1, const hevc_wp_t* wp, int ci) {
    if (!wp) return clip_u8((u0 && u1) ? (p0 + p1 + 64) >> 7 : ((u0 ? p0 : p1) + 32) >> 6);
    const int lw = wp->log2wd[ci ? 1 : 0];
    if (u0 && u1)
        return clip_u8((p0 * wp->w[0][ci] + p1 * wp->w[1][ci] + ((wp->o[0][ci] + wp->o[1][ci] + 1) << lw)) >> (lw + 1));
    const int l = u0 ? 0 : 1;
    return clip_u8((((u0 ? p0 : p1) * wp->w[l][ci] + (1 << (lw - 1))) >> lw) + wp->o[l][ci]);
}

// One list of one strip: NT-tap (8 luma, 4 chroma) prediction of 4 columns x h rows whose
// integer position is (xi, yi) with phases (fx, fy); emit(k, p) receives output row k.
template <int NT, typename Emit>
__device__ __forceinline__ void filter_strip(const uint8_t* plane, int pitch, int pw, int ph, int xi, int yi, int fx,
                                             int fy, int h, Emit&& emit) {
    constexpr int HALF = NT / 2 - 1;       // window starts HALF samples left / above
    constexpr int NW = NT == 8 ? 4 : 3;    // aligned words per window row
    const int x0 = xi - HALF, xa = x0 & ~3, sh = 8 * (x0 & 3), yw = yi - HALF;
    uint32_t tlo, thi = 0;
    int tv[NT];
    if constexpr (NT == 8) {
        tlo = c_luma_pk[fx][0];
        thi = c_luma_pk[fx][1];
        const uint32_t v0 = c_luma_pk[fy][0], v1 = c_luma_pk[fy][1];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            tv[q] = tap_of(v0, q);
            tv[q + 4] = tap_of(v1, q);
        }
    } else {
        tlo = c_chroma_pk[fx];
        const uint32_t v = c_chroma_pk[fy];
#pragma unroll
        for (int q = 0; q < 4; q++) tv[q] = tap_of(v, q);
    }
    const bool fast = x0 >= 0 && xa + 4 * NW <= pw && yw >= 0 && yw + h + NT - 1 <= ph;
    // horizontal filter of window row r into dst[0..3]
    auto hrow = [&](int r, int (&dst)[4]) {
        uint32_t w[NW];
        row_words<NW>(plane, pitch, pw, ph, yw + r, xa, fast, w);
        const uint32_t s0 = __funnelshift_r(w[0], w[1], sh), s1 = __funnelshift_r(w[1], w[2], sh);
        if constexpr (NT == 8) {
            const uint32_t s2 = __funnelshift_r(w[2], w[3], sh);
#pragma unroll
            for (int j = 0; j < 4; j++)
                dst[j] = dp4a_su(thi, __funnelshift_r(s1, s2, 8 * j), dp4a_su(tlo, __funnelshift_r(s0, s1, 8 * j), 0));
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) dst[j] = dp4a_su(tlo, __funnelshift_r(s0, s1, 8 * j), 0);
        }
    };
    // window row r lives in wnd[r % NT]: rows 0..NT-2 first, then groups of NT rows,
    // each adding window row g+NT-1+k and emitting output row g+k
    int wnd[NT][4];
#pragma unroll
    for (int r = 0; r < NT - 1; r++) hrow(r, wnd[r]);
#pragma unroll 1
    for (int g = 0; g < h; g += NT) {
#pragma unroll
        for (int k = 0; k < NT; k++) {
            if (g + k >= h) break;
            hrow(g + NT - 1 + k, wnd[(NT - 1 + k) % NT]);
            int p[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                int a = 0;
#pragma unroll
                for (int q = 0; q < NT; q++) a += tv[q] * wnd[(k + q) % NT][j];
                p[j] = a >> 6;
            }
            emit(g + k, p);
        }
    }
}

__device__ __forceinline__ uint32_t pack16(int a, int b) { return (uint32_t)(a & 0xFFFF) | ((uint32_t)b << 16); }
__device__ __forceinline__ int lo16(uint32_t v) { return (int)(int16_t)(v & 0xFFFF); }
__device__ __forceinline__ int hi16(uint32_t v) { return (int)(int16_t)(v >> 16); }

// One strip of one component: the lists run one after the other; a bi-predicted strip
// keeps its list-0 predictions in shared memory (s_pred[row][thread], int16 x 4) until the
// list-1 pass combines them.  Chroma strips may be 2 wide at the end of a 2/6-wide PU.
template <bool CHROMA>
__device__ __forceinline__ void mc_strip(const PicDesc& P, const hevc_pu_t& pu, const McStrip& s, uint2 (*s_pred)[MC_THREADS]) {
    const bool use0 = pu.ref_idx[0] >= 0, use1 = pu.ref_idx[1] >= 0, bi = use0 && use1;
    const hevc_wp_t* wp = pu.wp >= 0 ? &P.wp[pu.wp] : nullptr;
    const int tid = threadIdx.x;
    constexpr bool chroma = CHROMA;
    constexpr int sub = chroma ? 2 : 1;
    const int x = pu.x / sub + s.sx, y = pu.y / sub + s.sy, h = s.h;
    const int width = min(4, pu.w / sub - s.sx);
    const int pw = P.width / sub, ph = P.height / sub, pitch = chroma ? P.pitch_c : P.pitch_y;
#pragma unroll 1
    for (int ci = chroma ? 1 : 0; ci <= (chroma ? 2 : 0); ci++) {
        const int64_t poff = ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr);
        uint8_t* out = P.rec + poff + (int64_t)y * pitch + x;
#pragma unroll 1
        for (int pass = 0; pass < (bi ? 2 : 1); pass++) {
            const int l = bi ? pass : (use0 ? 0 : 1);
            const int mvx = pu.mv[l][0], mvy = pu.mv[l][1];
            const uint8_t* ref = P.ref[l][pu.ref_idx[l]] + poff;
            auto emit = [&](int k, const int (&p)[4]) {
                if (bi && pass == 0) {
                    s_pred[k][tid] = make_uint2(pack16(p[0], p[1]), pack16(p[2], p[3]));
                    return;
                }
                int q[4] = {p[0], p[1], p[2], p[3]};
                if (bi) {
                    const uint2 v = s_pred[k][tid];
                    q[0] = lo16(v.x); q[1] = hi16(v.x); q[2] = lo16(v.y); q[3] = hi16(v.y);
                }
                uint8_t* o = out + (int64_t)k * pitch;
                uint32_t b = 0;
#pragma unroll
                for (int j = 0; j < 4; j++) b |= (uint32_t)weigh(q[j], p[j], use0, use1, wp, ci) << (8 * j);
                if constexpr (!chroma) {
                    *reinterpret_cast<uint32_t*>(o) = b;   // luma strips are 4 wide and 4-aligned
                } else {
                    *reinterpret_cast<uint16_t*>(o) = (uint16_t)b;
                    if (width == 4) *reinterpret_cast<uint16_t*>(o + 2) = (uint16_t)(b >> 16);
                }
            };
            if constexpr (!chroma)
                filter_strip<8>(ref, pitch, pw, ph, x + (mvx >> 2), y + (mvy >> 2), mvx & 3, mvy & 3, h, emit);
            else
                filter_strip<4>(ref, pitch, pw, ph, x + (mvx >> 3), y + (mvy >> 3), mvx & 7, mvy & 7, h, emit);
        }
    }
}

// Luma strips and chroma strips are separate launches (separate item lists).
template <bool CHROMA>
__global__ void __launch_bounds__(MC_THREADS, 6) k_mc(const __grid_constant__ SegTable st) {
    __shared__ uint2 s_pred[16][MC_THREADS];
    const Seg& sg = st.s[find_seg(st, blockIdx.x)];
    const int item = (blockIdx.x - sg.block0) * MC_THREADS + threadIdx.x;
    if (item >= sg.n_items) return;
    const McStrip s = static_cast<const McStrip*>(sg.items)[item];
    const PicDesc& P = *sg.pic;
    const hevc_pu_t pu = P.pus[s.pu];
    mc_strip<CHROMA>(P, pu, s, s_pred);
}

}  // namespace hevcgpu
