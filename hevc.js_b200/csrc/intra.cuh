// intra.cuh — intra prediction (perform_intra_prediction, intra_prediction.cpp:428-481,
// with build_reference_samples :44-211, filtering :217-257, planar/DC/angular :263-422).
//
// Every intra TU reads reference samples left of and above it.  Those samples are final
// when this stage runs, except where an earlier intra TU writes them (MC and the inter
// residuals ran before).  The host turns that into a dependency list per intra TU: the
// TUs that write samples it reads, in its own CTU (local) or in an earlier CTU
// (external), and orders each CTU's TUs by their depth in the picture's dependency DAG.
// k_intra_ctus runs one CTA per CTU with intra TUs: it stages the CTU, its TU records,
// dependency lists and residuals in shared memory; its warps take the TUs in order and run
// each one once its dependencies are complete (one-arrival barriers in shared memory for
// local ones, published flags in global memory for external ones), reading samples of
// other CTUs from the picture through L2.  Every wait gives up after WAIT_LIMIT_NS of the
// GPU's global timer (or SPIN_LIMIT polls, should the timer not advance), sets ST_TIMEOUT
// in the context's sticky status word (the host turns it into HEVCGPU_ETIMEOUT) and
// returns.
#pragma once

#include <cuda/atomic>

#include "device_common.cuh"

namespace hevcgpu {

__constant__ int8_t c_intra_angle[35] = {0,   0,   32,  26,  21,  17,  13,  9,  5,  2,  0,  -2,
                                         -5,  -9,  -13, -17, -21, -26, -32, -26, -21, -17, -13, -9,
                                         -5,  -2,  0,   2,   5,   9,   13,  17,  21,  26,  32};
__constant__ int16_t c_inv_angle[35] = {0,    0,    256, 315, 390, 482,  630,  910,  1638, 4096, 0,   4096,
                                        1638, 910,  630, 482, 390, 315,  256,  315,  390,  482,  630, 910,
                                        1638, 4096, 0,   4096, 1638, 910, 630, 482,  390,  315,  256};

// The picture fields intra_tu reads, copied into shared memory once per CTA: reads of the
// descriptor in global memory would go through L1, which every GPU-scope acquire on the SM
// invalidates, and sit in each TU's chain of dependent loads.
struct IntraPic {
    uint8_t* rec;
    int64_t off_cb, off_cr;
    int32_t width, height, log2_ctb, pitch_y, pitch_c, intra_smoothing_disabled, strong_intra;
};

struct IntraWarpSmem {
    int16_t s[129];    // final references: bottom-left .. corner (index 2n) .. top-right
    int16_t m[130];    // angular main reference m[q + n], q = -n .. 2n (+1 padding entry)
};

// Shared-memory copy of one plane around the CTU being reconstructed: sample (x, y) of
// the plane is at t[(y - y0) * pitch + (x - x0)].
struct CtuTile {
    uint8_t* t;
    int pitch, x0, y0;
};

// Neighbour CTBs an intra TU may read from, as bits of a mask: they must precede the
// current CTB in raster order and share its slice and tile (intra_prediction.cpp:108-124).
enum : uint32_t { NB_LEFT = 1u, NB_ABOVE_LEFT = 2u, NB_ABOVE = 4u, NB_ABOVE_RIGHT = 8u };

// Predict + reconstruct one intra TU (any size 4..32, any plane) with one warp
// (perform_intra_prediction, then reconstruct_block's add and clip).  Reference samples
// come from the CTU tile, or from the picture for samples of other CTUs; results go to the
// tile (for later TUs) and the picture.  res is the TU's residual (null when it has none).
// The size is a run-time value: one copy of the code serves every TU, which keeps the
// kernel small in the instruction cache (TUs of every size alternate on an SM).  Between
// the lanes the reference array goes through the warp's shared memory.
template <typename Pic, typename Wait>
__device__ __forceinline__ bool intra_tu(const Pic& P, const hevc_tu_t& t, int lane, IntraWarpSmem& W,
                                         const CtuTile& tile, uint32_t nb_mask, const int16_t* res, Wait&& wait) {
    constexpr int RMAX = 5;                       // lane rounds of the largest reference array
    const int ci = t.c_idx, chroma = ci != 0, log2 = t.log2_size, n = 1 << log2, sub = chroma ? 2 : 1;
    const int total = 4 * n + 1, R = (total + 31) >> 5;   // reference samples, lane rounds
    const int xc = t.x, yc = t.y;
    const int log2c = P.log2_ctb - chroma;                // CTB size in this plane
    const int rx = xc >> log2c, ry = yc >> log2c;
    const int pw = P.width >> chroma, ph = P.height >> chroma;
    const int ox = rx << P.log2_ctb, oy = ry << P.log2_ctb;   // CTB origin in luma samples
    const int pitch = chroma ? P.pitch_c : P.pitch_y;
    uint8_t* plane = P.rec + (ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr));
    const uint32_t cur_z = zorder16((uint32_t)((xc * sub - ox) >> 2), (uint32_t)((yc * sub - oy) >> 2));

    // 1. reference samples and their availability: in the picture, and either in an
    //    earlier CTB of the same slice and tile, or in this CTB at a lower z-scan address
    //    of the 4x4 luma unit (intra_prediction.cpp:102-133).  Index i runs from the
    //    bottom-left sample (0) through the corner (2n) to the top-right one (4n).
    //    Availability and the address of each sample depend on positions only, so they are
    //    found before the wait for the TUs that write the samples; the loads follow it.
    uint32_t mask[RMAX];
    int val[RMAX], where[RMAX];   // where: tile index, or ~(picture offset) for samples of other CTUs
#pragma unroll
    for (int r = 0; r < RMAX; r++) {
        mask[r] = 0;
        where[r] = 0;
        if (r >= R) continue;
        const int i = lane + 32 * r;
        bool ok = false;
        int at = 0;
        if (i < total) {
            int px, py;
            if (i < 2 * n) { px = xc - 1; py = yc + 2 * n - 1 - i; }
            else if (i == 2 * n) { px = xc - 1; py = yc - 1; }
            else { px = xc + (i - 2 * n - 1); py = yc - 1; }
            if (px >= 0 && py >= 0 && px < pw && py < ph) {
                const int ncx = px >> log2c, ncy = py >> log2c;
                const bool outside = ncx != rx || ncy != ry;
                if (outside) {
                    // reference positions reach one CTB left, one CTB right (top row) and
                    // one CTB row up or down; later CTBs are never available
                    uint32_t bit = 0u;
                    if (ncy == ry) bit = ncx == rx - 1 ? NB_LEFT : 0u;
                    else if (ncy == ry - 1)
                        bit = ncx == rx - 1 ? NB_ABOVE_LEFT : (ncx == rx ? NB_ABOVE : (ncx == rx + 1 ? NB_ABOVE_RIGHT : 0u));
                    ok = (nb_mask & bit) != 0;
                } else {
                    ok = zorder16((uint32_t)((px * sub - ox) >> 2), (uint32_t)((py * sub - oy) >> 2)) < cur_z;
                }
                if (ok) at = outside ? ~(py * pitch + px) : (py - tile.y0) * tile.pitch + (px - tile.x0);
            }
        }
        where[r] = at;
        mask[r] = __ballot_sync(0xffffffffu, ok);
    }
    if (!wait()) return false;
    // samples of other CTUs come from the picture through L2 (the TUs of those CTUs that
    // write them have published their completion), this CTU's from the tile
#pragma unroll
    for (int r = 0; r < RMAX; r++) {
        int v = 0;
        if (r < R && ((mask[r] >> lane) & 1u)) v = where[r] < 0 ? __ldcg(plane + ~where[r]) : tile.t[where[r]];
        val[r] = v;
    }

    // 2. substitution (:177-197): an unavailable sample takes the nearest available one
    //    below it in the array, or the first available one; none available -> 128.  The
    //    raw samples go through W.m (free until step 4).
    const uint32_t last_lanes = (total & 31) ? ((1u << (total & 31)) - 1u) : 0xffffffffu;
    bool all = true;
    int first = -1;
#pragma unroll
    for (int r = 0; r < RMAX; r++) {
        if (r >= R) continue;
        all = all && mask[r] == (r == R - 1 ? last_lanes : 0xffffffffu);
        if (first < 0 && mask[r]) first = 32 * r + __ffs(mask[r]) - 1;
    }
    if (!all) {
        if (first >= 0) {
#pragma unroll
            for (int r = 0; r < RMAX; r++)
                if (r < R && lane + 32 * r < total) W.m[lane + 32 * r] = (int16_t)val[r];
            __syncwarp();
        }
#pragma unroll
        for (int r = 0; r < RMAX; r++) {
            if (r >= R) continue;
            if (first < 0) {
                val[r] = 128;
                continue;
            }
            if ((mask[r] >> lane) & 1u) continue;
            const uint32_t below = mask[r] & ((1u << lane) - 1u);
            int j = below ? 32 * r + 31 - __clz(below) : -1;
#pragma unroll
            for (int q = RMAX - 1; q >= 0; q--)
                if (q < r && j < 0 && mask[q]) j = 32 * q + 31 - __clz(mask[q]);
            val[r] = W.m[j < 0 ? first : j];
        }
    }
    // the substituted references to W.s
#pragma unroll
    for (int r = 0; r < RMAX; r++)
        if (r < R && lane + 32 * r < total) W.s[lane + 32 * r] = (int16_t)val[r];
    __syncwarp();

    // 3. smoothing of luma references (:217-257, :443-471): [1 2 1] over the linear array
    //    (which also gives the corner filter), or the bilinear strong smoothing of 32x32
    const int mode = t.intra_mode;
    if (!chroma && n != 4) {
        const int thr = n == 8 ? 7 : (n == 16 ? 1 : 0);
        const int d = min(abs(mode - 26), abs(mode - 10));
        if (!P.intra_smoothing_disabled && mode != 1 && d > thr) {
            const int c = W.s[2 * n], e_top = W.s[4 * n], e_left = W.s[0];
            const bool bil = n == 32 && P.strong_intra && abs(c + e_top - 2 * W.s[3 * n]) < 8 &&
                             abs(c + e_left - 2 * W.s[n]) < 8;
            int f[RMAX];
#pragma unroll
            for (int r = 0; r < RMAX; r++) {
                const int i = lane + 32 * r;
                f[r] = val[r];
                if (r >= R || i == 0 || i >= 4 * n) continue;
                if (bil) {
                    if (i > 2 * n) { const int k = i - 2 * n; f[r] = ((2 * n - k) * c + k * e_top + n) >> (log2 + 1); }
                    else if (i < 2 * n) { const int k = 2 * n - i; f[r] = ((2 * n - k) * c + k * e_left + n) >> (log2 + 1); }
                } else {
                    f[r] = (W.s[i - 1] + 2 * val[r] + W.s[i + 1] + 2) >> 2;
                }
            }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < RMAX; r++)
                if (r < R && lane + 32 * r < total) W.s[lane + 32 * r] = (int16_t)f[r];
            __syncwarp();
        }
    }
    // 4. for the angular modes, the main reference with the side reference projected
    //    through invAngle (:346-368): m[q + n] = top[q] (vertical) / left[q] (horizontal)
    //    for q >= 0, the other side's sample min(2n, (-q * invAngle + 128) >> 8) for q < 0
    //    (top[k] = R_[2n + k], left[k] = R_[2n - k])
    const int16_t* R_ = W.s;
    const int ang = c_intra_angle[mode];
    const bool vert = mode >= 18;
    if (mode >= 2) {
        const int inv = c_inv_angle[mode];
        const int me = 3 * n + 2;   // entries q = -n .. 2n + 1 (the last one padding, never weighted)
        for (int e = lane; e < me; e += 32) {
            const int q = e - n;
            int src;
            if (q > 2 * n) src = -1;
            else if (q >= 0) src = vert ? 2 * n + q : 2 * n - q;
            else {
                const int si = min(2 * n, ((-q) * inv + 128) >> 8);
                src = vert ? 2 * n - si : 2 * n + si;
            }
            W.m[e] = src < 0 ? (int16_t)0 : R_[src];
        }
        __syncwarp();
    }
    // 5. prediction + residual, clip, store.  Each lane takes groups of 4 samples of a row;
    //    its column x0 = 4 * (lane % (n / 4)) is the same for all its groups, so column
    //    terms are computed once.
    const int gpr = n >> 2, ng = (n * n) >> 2;
    int dc = 0;
    if (mode == 1) {  // predict_dc :295-317
        int sum = 0;
        for (int i = lane; i < n; i += 32) sum += R_[2 * n + 1 + i] + R_[2 * n - 1 - i];
        sum = __reduce_add_sync(0xffffffffu, sum);
        dc = (sum + n) >> (log2 + 1);
    }
    const int x0 = 4 * (lane & (gpr - 1));
    const int corner = R_[2 * n], tr = R_[3 * n + 1], bl = R_[n - 1];
    int ctop[4], cidx[4], cfr[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int x = x0 + j;
        ctop[j] = R_[2 * n + 1 + x];
        cidx[j] = ((x + 1) * ang) >> 5;
        cfr[j] = ((x + 1) * ang) & 31;
    }
    const bool edge_filters = !chroma && n < 32;
    for (int g = lane; g < ng; g += 32) {
        const int y = g >> (log2 - 2);
        const int left = R_[2 * n - 1 - y];
        int p[4];
        if (mode == 0) {  // predict_planar :263-289
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int x = x0 + j;
                p[j] = ((n - 1 - x) * left + (x + 1) * tr + (n - 1 - y) * ctop[j] + (y + 1) * bl + n) >> (log2 + 1);
            }
        } else if (mode == 1) {
#pragma unroll
            for (int j = 0; j < 4; j++) p[j] = dc;
            if (edge_filters) {
                if (y == 0) {
#pragma unroll
                    for (int j = 0; j < 4; j++) p[j] = (ctop[j] + 3 * dc + 2) >> 2;
                }
                if (x0 == 0) p[0] = y == 0 ? (ctop[0] + left + 2 * dc + 2) >> 2 : (left + 3 * dc + 2) >> 2;
            }
        } else if (vert) {  // predict_angular :323-422, main reference on top
            const int idx = ((y + 1) * ang) >> 5, fr = ((y + 1) * ang) & 31;
            const int16_t* m = W.m + n + x0 + 1 + idx;
            int r5[5];
#pragma unroll
            for (int j = 0; j < 5; j++) r5[j] = m[j];
#pragma unroll
            for (int j = 0; j < 4; j++) p[j] = fr ? ((32 - fr) * r5[j] + fr * r5[j + 1] + 16) >> 5 : r5[j];
            if (edge_filters && mode == 26 && x0 == 0) p[0] = clip_u8(p[0] + ((left - corner) >> 1));
        } else {  // main reference on the left
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int16_t* m = W.m + n + y + 1 + cidx[j];
                p[j] = cfr[j] ? ((32 - cfr[j]) * m[0] + cfr[j] * m[1] + 16) >> 5 : m[0];
            }
            if (edge_filters && mode == 10 && y == 0) {
#pragma unroll
                for (int j = 0; j < 4; j++) p[j] = clip_u8(p[j] + ((ctop[j] - corner) >> 1));
            }
        }
        if (t.flags & HEVC_TU_PCM) {   // the PCM samples are the levels, with no prediction
#pragma unroll
            for (int j = 0; j < 4; j++) p[j] = 0;
        }
        // residual (four int16 in one 8-byte load), clip, one word to the tile and the picture
        int rv[4] = {0, 0, 0, 0};
        if (res) {
            const int2 rw = *reinterpret_cast<const int2*>(res + y * n + x0);
            rv[0] = (int)(int16_t)(rw.x & 0xFFFF);
            rv[1] = rw.x >> 16;
            rv[2] = (int)(int16_t)(rw.y & 0xFFFF);
            rv[3] = rw.y >> 16;
        }
        uint32_t w = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) w |= (uint32_t)clip_u8(p[j] + rv[j]) << (8 * j);
        *reinterpret_cast<uint32_t*>(tile.t + (yc + y - tile.y0) * tile.pitch + (xc + x0 - tile.x0)) = w;
        *reinterpret_cast<uint32_t*>(plane + (int64_t)(yc + y) * pitch + xc + x0) = w;
    }
    return true;
}

// The 4x4 TU (luma or chroma; most TUs, and most of an intra picture's dependency chain):
// the same prediction with the 17 reference samples held one per lane and moved by
// shuffles, no smoothing (4x4 references are never filtered, :217-230 and :443-445), and one
// output sample per lane (x = lane & 3, y = lane >> 2) — no shared-memory staging.
template <typename Pic, typename Wait>
__device__ __forceinline__ bool intra_tu4(const Pic& P, const hevc_tu_t& t, int lane, const CtuTile& tile,
                                          uint32_t nb_mask, const int16_t* res, Wait&& wait) {
    constexpr uint32_t FULL = 0xffffffffu, ALL17 = 0x1FFFFu;
    const int ci = t.c_idx, chroma = ci != 0, sub = chroma ? 2 : 1;
    const int xc = t.x, yc = t.y;
    const int log2c = P.log2_ctb - chroma;
    const int rx = xc >> log2c, ry = yc >> log2c;
    const int pw = P.width >> chroma, ph = P.height >> chroma;
    const int ox = rx << P.log2_ctb, oy = ry << P.log2_ctb;
    const int pitch = chroma ? P.pitch_c : P.pitch_y;
    uint8_t* plane = P.rec + (ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr));
    // 1. reference sample `lane` (0 bottom-left .. 8 corner .. 16 top-right), its availability
    //    (intra_prediction.cpp:102-133) and where it lies, before the wait
    bool ok = false;
    int at = 0;
    if (lane < 17) {
        int px, py;
        if (lane < 8) { px = xc - 1; py = yc + 7 - lane; }
        else if (lane == 8) { px = xc - 1; py = yc - 1; }
        else { px = xc + lane - 9; py = yc - 1; }
        if (px >= 0 && py >= 0 && px < pw && py < ph) {
            const int ncx = px >> log2c, ncy = py >> log2c;
            const bool outside = ncx != rx || ncy != ry;
            if (outside) {
                uint32_t bit = 0u;
                if (ncy == ry) bit = ncx == rx - 1 ? NB_LEFT : 0u;
                else if (ncy == ry - 1)
                    bit = ncx == rx - 1 ? NB_ABOVE_LEFT : (ncx == rx ? NB_ABOVE : (ncx == rx + 1 ? NB_ABOVE_RIGHT : 0u));
                ok = (nb_mask & bit) != 0;
            } else {
                const uint32_t cur_z = zorder16((uint32_t)((xc * sub - ox) >> 2), (uint32_t)((yc * sub - oy) >> 2));
                ok = zorder16((uint32_t)((px * sub - ox) >> 2), (uint32_t)((py * sub - oy) >> 2)) < cur_z;
            }
            if (ok) at = outside ? ~(py * pitch + px) : (py - tile.y0) * tile.pitch + (px - tile.x0);
        }
    }
    const uint32_t mask = __ballot_sync(FULL, ok);
    if (!wait()) return false;
    int v = ok ? (at < 0 ? (int)__ldcg(plane + ~at) : (int)tile.t[at]) : 0;
    // 2. substitution (:177-197): the nearest available sample below, else the first one;
    //    none available -> 128
    if (mask != ALL17) {
        const uint32_t below = mask & ((1u << lane) - 1u);
        const int j = ((mask >> lane) & 1u) ? lane : (below ? 31 - __clz(below) : __ffs(mask) - 1);
        v = __shfl_sync(FULL, v, j < 0 ? 0 : j);
        if (mask == 0u) v = 128;
    }
    // 3. prediction of sample (x, y) of this lane (planar :263-289, DC :295-317, angular
    //    :323-422 with the main reference projected through invAngle :346-368)
    const int x = lane & 3, y = (lane >> 2) & 3, mode = t.intra_mode;
    const int left = __shfl_sync(FULL, v, 7 - y), top = __shfl_sync(FULL, v, 9 + x);
    const int corner = __shfl_sync(FULL, v, 8);
    int p;
    if (mode == 0) {
        const int tr = __shfl_sync(FULL, v, 13), bl = __shfl_sync(FULL, v, 3);
        p = ((3 - x) * left + (x + 1) * tr + (3 - y) * top + (y + 1) * bl + 4) >> 3;
    } else if (mode == 1) {
        const int dc = (__reduce_add_sync(FULL, ((lane >= 4 && lane <= 7) || (lane >= 9 && lane <= 12)) ? v : 0) + 4) >> 3;
        p = dc;
        if (!chroma) {
            if (y == 0) p = x == 0 ? (top + left + 2 * dc + 2) >> 2 : (top + 3 * dc + 2) >> 2;
            else if (x == 0) p = (left + 3 * dc + 2) >> 2;
        }
    } else {
        const bool vert = mode >= 18;
        const int ang = c_intra_angle[mode], inv = c_inv_angle[mode];
        const int along = vert ? y : x, across = vert ? x : y;
        const int idx = ((along + 1) * ang) >> 5, fr = ((along + 1) * ang) & 31;
        // main reference entry q (q >= 0: the main side; q < 0: the other side projected)
        auto src = [&](int q) {
            int s;
            if (q >= 0) s = vert ? 8 + q : 8 - q;
            else {
                const int si = min(8, ((-q) * inv + 128) >> 8);
                s = vert ? 8 - si : 8 + si;
            }
            return min(16, max(0, s));   // past the end only with weight 0
        };
        const int q = across + 1 + idx;
        const int a = __shfl_sync(FULL, v, src(q)), b = __shfl_sync(FULL, v, src(q + 1));
        p = fr ? ((32 - fr) * a + fr * b + 16) >> 5 : a;
        if (!chroma && mode == 26 && x == 0) p = clip_u8(p + ((left - corner) >> 1));
        if (!chroma && mode == 10 && y == 0) p = clip_u8(p + ((top - corner) >> 1));
    }
    if (t.flags & HEVC_TU_PCM) p = 0;   // the PCM samples are the levels, with no prediction
    if (lane < 16) {
        const uint8_t o = (uint8_t)clip_u8(p + (res ? res[lane] : 0));
        tile.t[(yc + y - tile.y0) * tile.pitch + (xc + x - tile.x0)] = o;
        plane[(int64_t)(yc + y) * pitch + xc + x] = o;
    }
    return true;
}

// The 8x8 TU: the same prediction as intra_tu with its 33 reference samples in registers,
// sample k in lane k for k < 32 and the last one (the far end of the top row) held by every
// lane, moved by shuffles; luma smoothing (:217-257, 8x8 threshold 7) with the lanes'
// neighbours; two output samples per lane, (x, y) and (x, y + 4) with x = lane & 7 and
// y = lane >> 3.
template <typename Pic, typename Wait>
__device__ __forceinline__ bool intra_tu8(const Pic& P, const hevc_tu_t& t, int lane, const CtuTile& tile,
                                          uint32_t nb_mask, const int16_t* res, Wait&& wait) {
    constexpr uint32_t FULL = 0xffffffffu;
    const int ci = t.c_idx, chroma = ci != 0, sub = chroma ? 2 : 1;
    const int xc = t.x, yc = t.y;
    const int log2c = P.log2_ctb - chroma;
    const int rx = xc >> log2c, ry = yc >> log2c;
    const int pw = P.width >> chroma, ph = P.height >> chroma;
    const int ox = rx << P.log2_ctb, oy = ry << P.log2_ctb;
    const int pitch = chroma ? P.pitch_c : P.pitch_y;
    uint8_t* plane = P.rec + (ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr));
    const uint32_t cur_z = zorder16((uint32_t)((xc * sub - ox) >> 2), (uint32_t)((yc * sub - oy) >> 2));
    // 1. reference sample k (0 bottom-left .. 16 corner .. 32 top-right), its availability
    //    (intra_prediction.cpp:102-133) and where it lies, before the wait
    auto locate = [&](int k, int& at) -> bool {
        int px, py;
        if (k < 16) { px = xc - 1; py = yc + 15 - k; }
        else if (k == 16) { px = xc - 1; py = yc - 1; }
        else { px = xc + k - 17; py = yc - 1; }
        if (px < 0 || py < 0 || px >= pw || py >= ph) return false;
        const int ncx = px >> log2c, ncy = py >> log2c;
        const bool outside = ncx != rx || ncy != ry;
        bool ok;
        if (outside) {
            uint32_t bit = 0u;
            if (ncy == ry) bit = ncx == rx - 1 ? NB_LEFT : 0u;
            else if (ncy == ry - 1)
                bit = ncx == rx - 1 ? NB_ABOVE_LEFT : (ncx == rx ? NB_ABOVE : (ncx == rx + 1 ? NB_ABOVE_RIGHT : 0u));
            ok = (nb_mask & bit) != 0;
        } else {
            ok = zorder16((uint32_t)((px * sub - ox) >> 2), (uint32_t)((py * sub - oy) >> 2)) < cur_z;
        }
        if (ok) at = outside ? ~(py * pitch + px) : (py - tile.y0) * tile.pitch + (px - tile.x0);
        return ok;
    };
    int at = 0, at32 = 0;
    const bool ok = locate(lane, at);
    const bool ok32 = locate(32, at32);   // the same in every lane
    const uint32_t mask = __ballot_sync(FULL, ok);
    // substitution (:177-197) as a map from k to the sample it takes: k itself when
    // available, else the nearest available one below, else the first available one; 32 is
    // the last entry.  None available: every sample is 128.
    const bool none = mask == 0u && !ok32;
    auto sl = [&](int k) -> int {
        if (k == 32) return ok32 ? 32 : (mask ? 31 - __clz(mask) : 32);
        if ((mask >> k) & 1u) return k;
        const uint32_t below = mask & ((1u << k) - 1u);
        return below ? 31 - __clz(below) : (mask ? __ffs(mask) - 1 : 32);
    };
    const int mode = t.intra_mode;
    const int x = lane & 7, y0 = lane >> 3;
    const bool smooth = !chroma && !P.intra_smoothing_disabled && mode != 1 && min(abs(mode - 26), abs(mode - 10)) > 7;
    const int own = sl(lane), own_prev = sl(max(lane - 1, 0)), own_next = sl(lane + 1);
    const int rv0 = res != nullptr ? res[y0 * 8 + x] : 0, rv1 = res != nullptr ? res[(y0 + 4) * 8 + x] : 0;
    if (!wait()) return false;
    // 2. the samples, substituted: lane k holds R[k] (k < 32), every lane R[32]
    const int raw = ok ? (at < 0 ? (int)__ldcg(plane + ~at) : (int)tile.t[at]) : 0;
    const int raw32 = ok32 ? (at32 < 0 ? (int)__ldcg(plane + ~at32) : (int)tile.t[at32]) : 0;
    auto take = [&](int j) { const int v = __shfl_sync(FULL, raw, j & 31); return j == 32 ? raw32 : v; };
    int r = none ? 128 : take(own);
    int r32 = none ? 128 : take(sl(32));
    // 3. smoothing of luma references: [1 2 1] over the linear array, ends kept
    if (smooth) {
        const int prev = none ? 128 : take(own_prev), next = none ? 128 : take(own_next);
        r = lane == 0 ? r : (prev + 2 * r + next + 2) >> 2;
    }
    // 4. prediction of (x, y0) and (x, y0 + 4)
    auto R = [&](int k) { const int v = __shfl_sync(FULL, r, k & 31); return k >= 32 ? r32 : v; };
    int p[2];
    if (mode == 0) {   // planar (:263-289)
        const int tr = R(25), bl = R(7), top = R(17 + x);
        const int l0 = R(15 - y0), l1 = R(11 - y0);
        p[0] = ((7 - x) * l0 + (x + 1) * tr + (7 - y0) * top + (y0 + 1) * bl + 8) >> 4;
        p[1] = ((7 - x) * l1 + (x + 1) * tr + (3 - y0) * top + (y0 + 5) * bl + 8) >> 4;
    } else if (mode == 1) {   // DC (:295-317): left R[8..15], top R[17..24]
        const bool in_sum = (lane >= 8 && lane <= 15) || (lane >= 17 && lane <= 24);
        const int dc = (__reduce_add_sync(FULL, in_sum ? r : 0) + 8) >> 4;
        const int top = R(17 + x), l0 = R(15 - y0), l1 = R(11 - y0);
        p[0] = dc;
        p[1] = dc;
        if (!chroma) {
            if (y0 == 0) p[0] = x == 0 ? (top + l0 + 2 * dc + 2) >> 2 : (top + 3 * dc + 2) >> 2;
            else if (x == 0) p[0] = (l0 + 3 * dc + 2) >> 2;
            if (x == 0) p[1] = (l1 + 3 * dc + 2) >> 2;
        }
    } else {   // angular (:323-422), main reference projected through invAngle (:346-368)
        const bool vert = mode >= 18;
        const int ang = c_intra_angle[mode], inv = c_inv_angle[mode];
        auto src = [&](int q) {
            int s;
            if (q >= 0) s = vert ? 16 + q : 16 - q;
            else {
                const int si = min(16, ((-q) * inv + 128) >> 8);
                s = vert ? 16 - si : 16 + si;
            }
            return min(32, max(0, s));   // past the end only with weight 0
        };
        const int corner = R(16);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int y = y0 + 4 * h;
            const int along = vert ? y : x, across = vert ? x : y;
            const int idx = ((along + 1) * ang) >> 5, fr = ((along + 1) * ang) & 31;
            const int q = across + 1 + idx;
            // every shuffle by all lanes: left and top are read before the lane-dependent tests
            const int a = R(src(q)), b = R(src(q + 1)), left = R(15 - y), top = R(17 + x);
            int v = ((32 - fr) * a + fr * b + 16) >> 5;
            if (!chroma && mode == 26 && x == 0) v = clip_u8(v + ((left - corner) >> 1));
            if (!chroma && mode == 10 && y == 0) v = clip_u8(v + ((top - corner) >> 1));
            p[h] = v;
        }
    }
    if (t.flags & HEVC_TU_PCM) p[0] = p[1] = 0;   // the PCM samples are the levels, with no prediction
    const uint8_t o0 = (uint8_t)clip_u8(p[0] + rv0), o1 = (uint8_t)clip_u8(p[1] + rv1);
    tile.t[(yc + y0 - tile.y0) * tile.pitch + (xc + x - tile.x0)] = o0;
    tile.t[(yc + y0 + 4 - tile.y0) * tile.pitch + (xc + x - tile.x0)] = o1;
    plane[(int64_t)(yc + y0) * pitch + xc + x] = o0;
    plane[(int64_t)(yc + y0 + 4) * pitch + xc + x] = o1;
    return true;
}

// The 16x16 TU: its 65 reference samples in registers for substitution and smoothing,
// samples k and k + 32 in lane k (k < 32) and the last one (the far end of the top row) in
// every lane, moved by shuffles; then the final array in the warp's shared memory, from
// which each lane predicts (x, y) for x = lane & 15 and y = (lane >> 4) + 2i, i < 8, the
// angular ones straight from the reference array through invAngle (no projected copy).
template <typename Pic, typename Wait>
__device__ __forceinline__ bool intra_tu16(const Pic& P, const hevc_tu_t& t, int lane, IntraWarpSmem& W,
                                           const CtuTile& tile, uint32_t nb_mask, const int16_t* res, Wait&& wait) {
    constexpr uint32_t FULL = 0xffffffffu;
    const int ci = t.c_idx, chroma = ci != 0, sub = chroma ? 2 : 1;
    const int xc = t.x, yc = t.y;
    const int log2c = P.log2_ctb - chroma;
    const int rx = xc >> log2c, ry = yc >> log2c;
    const int pw = P.width >> chroma, ph = P.height >> chroma;
    const int ox = rx << P.log2_ctb, oy = ry << P.log2_ctb;
    const int pitch = chroma ? P.pitch_c : P.pitch_y;
    uint8_t* plane = P.rec + (ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr));
    const uint32_t cur_z = zorder16((uint32_t)((xc * sub - ox) >> 2), (uint32_t)((yc * sub - oy) >> 2));
    // 1. reference sample k (0 bottom-left .. 32 corner .. 64 top-right), its availability
    //    (intra_prediction.cpp:102-133) and where it lies, before the wait
    auto locate = [&](int k, int& at) -> bool {
        int px, py;
        if (k < 32) { px = xc - 1; py = yc + 31 - k; }
        else if (k == 32) { px = xc - 1; py = yc - 1; }
        else { px = xc + k - 33; py = yc - 1; }
        if (px < 0 || py < 0 || px >= pw || py >= ph) return false;
        const int ncx = px >> log2c, ncy = py >> log2c;
        const bool outside = ncx != rx || ncy != ry;
        bool ok;
        if (outside) {
            uint32_t bit = 0u;
            if (ncy == ry) bit = ncx == rx - 1 ? NB_LEFT : 0u;
            else if (ncy == ry - 1)
                bit = ncx == rx - 1 ? NB_ABOVE_LEFT : (ncx == rx ? NB_ABOVE : (ncx == rx + 1 ? NB_ABOVE_RIGHT : 0u));
            ok = (nb_mask & bit) != 0;
        } else {
            ok = zorder16((uint32_t)((px * sub - ox) >> 2), (uint32_t)((py * sub - oy) >> 2)) < cur_z;
        }
        if (ok) at = outside ? ~(py * pitch + px) : (py - tile.y0) * tile.pitch + (px - tile.x0);
        return ok;
    };
    int at_a = 0, at_b = 0, at64 = 0;
    const bool ok_a = locate(lane, at_a), ok_b = locate(lane + 32, at_b);
    const bool ok64 = locate(64, at64);   // the same in every lane
    const uint32_t m0 = __ballot_sync(FULL, ok_a), m1 = __ballot_sync(FULL, ok_b);
    // substitution (:177-197) as a map from k to the sample it takes: k itself when
    // available, else the nearest available one below, else the first available one.
    // None available: every sample is 128.
    const bool none = m0 == 0u && m1 == 0u && !ok64;
    auto sl = [&](int k) -> int {
        const bool av = k < 32 ? ((m0 >> k) & 1u) != 0 : (k < 64 ? ((m1 >> (k - 32)) & 1u) != 0 : ok64);
        if (av) return k;
        if (k > 32) {
            const uint32_t b1 = k >= 64 ? m1 : (m1 & ((1u << (k - 32)) - 1u));
            if (b1) return 63 - __clz(b1);
        }
        const uint32_t b0 = k >= 32 ? m0 : (m0 & ((1u << k) - 1u));
        if (b0) return 31 - __clz(b0);
        if (m0) return __ffs(m0) - 1;
        if (m1) return 31 + __ffs(m1);
        return 64;
    };
    const int mode = t.intra_mode;
    const bool smooth = !chroma && !P.intra_smoothing_disabled && mode != 1 && min(abs(mode - 26), abs(mode - 10)) > 1;
    const int ja = sl(lane), jb = sl(lane + 32), j64 = sl(64);
    if (!wait()) return false;
    // 2. the samples, substituted: lane k holds R[k] and R[k + 32], every lane R[64]
    auto load = [&](bool ok, int at) { return ok ? (at < 0 ? (int)__ldcg(plane + ~at) : (int)tile.t[at]) : 0; };
    const int raw_a = load(ok_a, at_a), raw_b = load(ok_b, at_b), raw64 = load(ok64, at64);
    auto take = [&](int j) {
        const int va = __shfl_sync(FULL, raw_a, j & 31), vb = __shfl_sync(FULL, raw_b, j & 31);
        return j < 32 ? va : (j < 64 ? vb : raw64);
    };
    int ra = none ? 128 : take(ja), rb = none ? 128 : take(jb);
    const int r64 = none ? 128 : take(j64);
    // 3. smoothing of luma references (:217-257, 16x16 threshold 1): [1 2 1] over the linear
    //    array, ends kept; the neighbours by shuffles of all lanes
    if (smooth) {
        const int up_a = __shfl_sync(FULL, ra, (lane + 31) & 31), dn_a = __shfl_sync(FULL, ra, (lane + 1) & 31);
        const int up_b = __shfl_sync(FULL, rb, (lane + 31) & 31), dn_b = __shfl_sync(FULL, rb, (lane + 1) & 31);
        const int next_a = lane < 31 ? dn_a : dn_b;            // lane 31: R[32], lane 0's rb
        const int prev_b = lane > 0 ? up_b : up_a;             // lane 0: R[31], lane 31's ra
        const int next_b = lane < 31 ? dn_b : r64;
        const int fa = lane == 0 ? ra : (up_a + 2 * ra + next_a + 2) >> 2;
        rb = (prev_b + 2 * rb + next_b + 2) >> 2;
        ra = fa;
    }
    W.s[lane] = (int16_t)ra;
    W.s[32 + lane] = (int16_t)rb;
    if (lane == 0) W.s[64] = (int16_t)r64;
    __syncwarp();
    // 4. prediction, residual, clip, store: (x, y) for y = (lane >> 4) + 2i
    const int16_t* Rs = W.s;
    const int x = lane & 15, ys = lane >> 4;
    const int corner = Rs[32], top_x = Rs[33 + x];
    int dc = 0;
    if (mode == 1) {   // DC (:295-317): left R[16..31], top R[33..48]
        const int part = (lane >= 16 ? ra : 0) + (lane >= 1 && lane <= 16 ? rb : 0);
        dc = (__reduce_add_sync(FULL, part) + 16) >> 5;
    }
    const bool vert = mode >= 18;
    const int ang = c_intra_angle[mode], inv = c_inv_angle[mode];
    auto src = [&](int q) {
        int s;
        if (q >= 0) s = vert ? 32 + q : 32 - q;
        else {
            const int si = min(32, ((-q) * inv + 128) >> 8);
            s = vert ? 32 - si : 32 + si;
        }
        return min(64, max(0, s));   // past the end only with weight 0
    };
    const bool pcm = (t.flags & HEVC_TU_PCM) != 0;   // the PCM samples are the levels, with no prediction
#pragma unroll 2
    for (int i = 0; i < 8; i++) {
        const int y = ys + 2 * i;
        const int left = Rs[31 - y];
        int p;
        if (mode == 0) {   // planar (:263-289)
            p = ((15 - x) * left + (x + 1) * Rs[49] + (15 - y) * top_x + (y + 1) * Rs[15] + 16) >> 5;
        } else if (mode == 1) {
            p = dc;
            if (!chroma) {
                if (y == 0) p = x == 0 ? (top_x + left + 2 * dc + 2) >> 2 : (top_x + 3 * dc + 2) >> 2;
                else if (x == 0) p = (left + 3 * dc + 2) >> 2;
            }
        } else {   // angular (:323-422)
            const int along = vert ? y : x, across = vert ? x : y;
            const int idx = ((along + 1) * ang) >> 5, fr = ((along + 1) * ang) & 31;
            const int q = across + 1 + idx;
            p = ((32 - fr) * Rs[src(q)] + fr * Rs[src(q + 1)] + 16) >> 5;
            if (!chroma && mode == 26 && x == 0) p = clip_u8(p + ((left - corner) >> 1));
            if (!chroma && mode == 10 && y == 0) p = clip_u8(p + ((top_x - corner) >> 1));
        }
        if (pcm) p = 0;
        const uint8_t o = (uint8_t)clip_u8(p + (res != nullptr ? res[y * 16 + x] : 0));
        tile.t[(yc + y - tile.y0) * tile.pitch + (xc + x - tile.x0)] = o;
        plane[(int64_t)(yc + y) * pitch + xc + x] = o;
    }
    return true;
}

// ---------------------------------------------------------------------------------------
// CTU tasks.  One CTA per CTU that holds intra TUs.  CTAs take CTUs by ticket in wavefront
// order per picture (2 * row + column: the diagonal band along which a picture's
// dependencies advance), the pictures of a launch side by side.  The CTA stages the CTU, its TU
// records and their residuals in shared memory; then its warps take the TUs one at a time
// in task order (by depth in the picture's DAG, so every TU comes after the TUs it depends
// on) and run each as soon as the TUs it reads from are complete: a TU of the same CTU
// through its one-arrival barrier in shared memory, a TU of an earlier CTU through that
// TU's published completion in global memory.  No barrier ties the warps together, so the
// critical path is the chain of dependent TUs itself.  Every wait is for a TU taken
// earlier, by this CTA or by a CTA holding an earlier ticket, which is already running;
// every wait is bounded.  The CTA's last warp is its watcher: it alone polls the global
// flags of the TUs of other CTUs, so the workers only wait on shared-memory barriers, which
// suspend them without taking issue slots.
// ---------------------------------------------------------------------------------------
constexpr int IC_WARPS = 8;
constexpr int IC_THREADS = 32 * IC_WARPS;
constexpr int IC_MIN_BLOCKS = 3;
constexpr int IC_LP = 64, IC_LH = 64;                // luma tile (the CTU): pitch, rows
constexpr int IC_CP = 32, IC_CH = 32;                // chroma tiles
constexpr int IC_MAX_TUS = 256 + 2 * 64;             // 4x4 TUs of a 64x64 CTU, all planes
constexpr int IC_MAX_RES = 64 * 64 + 2 * 32 * 32;    // residual samples of a 64x64 CTU
constexpr int IC_DEP_STAGE = 2048;                   // dependency entries staged per CTU
constexpr int IC_MAX_WATCH = 128;                    // TUs of other CTUs a CTU waits for
constexpr int IC_WATCHER = IC_WARPS - 1;             // the warp that watches them
constexpr unsigned long long WAIT_LIMIT_NS = 1000000000ull;   // a wait gives up after a second
constexpr unsigned SPIN_LIMIT = 1u << 26;            // backstop: polls of at least 64 ns

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// 16-byte asynchronous global -> shared copy (through L2 only, so that samples other
// CTUs wrote are seen), and the wait for all of a thread's copies.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// One-arrival barriers in shared memory, one per TU of the CTU: the warp that completes
// the TU arrives (release), the warps whose TUs read its samples wait on phase 0 (acquire).
// A waiting thread is suspended by the hardware until the phase completes or the time hint
// runs out, so waiting warps take no issue slots from the working ones.
__device__ __forceinline__ void mbar_init1(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(bar))
                 : "memory");
}
// true once phase 0 of the barrier has completed; false when the time hint ran out first
__device__ __forceinline__ bool mbar_try_wait0(uint64_t* bar) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], 0, %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"((uint32_t)__cvta_generic_to_shared(bar)), "r"(20000u)
        : "memory");
    return ok != 0;
}

// Copy plane c of CTU (rx, ry) into its tile with 16-byte copies (issued, not waited
// for).  Only the CTU itself: reference samples of other CTUs are read from the picture.
__device__ __forceinline__ void stage_tile(const PicDesc& P, int c, int rx, int ry, uint8_t* tile, int tid) {
    const int sub = c ? 2 : 1, ctbc = (1 << P.log2_ctb) / sub;
    const int pw = P.width / sub, ph = P.height / sub, pitch = c ? P.pitch_c : P.pitch_y;
    const uint8_t* plane = P.rec + (c == 0 ? 0 : (c == 1 ? P.off_cb : P.off_cr));
    const int tp = c ? IC_CP : IC_LP;
    const int x0 = rx * ctbc, y0 = ry * ctbc;
    if (ctbc >= 16) {
        const int row_chunks = ctbc / 16;
        for (int e = tid; e < ctbc * row_chunks; e += IC_THREADS) {
            const int r = e / row_chunks, q = e % row_chunks;
            const int y = y0 + r, x = x0 + 16 * q;
            if (y >= ph || x >= pw) continue;
            cp_async16(tile + r * tp + 16 * q, plane + (int64_t)y * pitch + x);
        }
    } else {  // 8-sample chroma CTBs (16x16 CTUs): words
        for (int e = tid; e < ctbc * 2; e += IC_THREADS) {
            const int r = e / 2, q = e % 2;
            const int y = y0 + r, x = x0 + 4 * q;
            if (y >= ph || x >= pw) continue;
            *reinterpret_cast<uint32_t*>(tile + r * tp + 4 * q) =
                __ldcg(reinterpret_cast<const uint32_t*>(plane + (int64_t)y * pitch + x));
        }
    }
}

// The state one worker's wait for a TU's dependencies reads.
struct IntraWait {
    const uint32_t* s_dep;      // the CTU's staged dependency entries
    const uint32_t* dep_list;   // all entries (those past the staged ones)
    uint64_t* s_bar;            // completion barriers of the CTU's TUs
    uint64_t* s_wbar;           // watch barriers
    int32_t* itu_done;          // published completions (direct external entries)
    uint32_t* sticky;
    volatile int* s_abort;
    int dfirst, doff, dcount, staged, task, n_watch, n_itu, epoch, lane;
};

// The wait for a TU's dependencies, between the position work and the loads of a TU path.
// Local and watched entries wait on shared-memory barriers; a direct external entry (only a
// planted test wait has one) polls the published completion.  Every wait reads the global
// timer and gives up after WAIT_LIMIT_NS (SPIN_LIMIT tries as a backstop), marking the
// sticky status; a wait also ends when another warp of the CTA gave up (s_abort) or, for
// external waits, when a wait anywhere did (the status word).  Inlined into the four TU
// paths: as a call it passed its arguments through the stack and saved and restored
// registers around every wait, on the critical path of each dependency step.
__device__ __forceinline__ bool intra_wait(const IntraWait& w) {
    // The entries one after another, every lane on the same one (warp-uniform waits: the
    // warp is suspended as a whole on a barrier).
    bool gave_up = false;
    for (int q = 0; q < w.dcount && !gave_up; q++) {
        const int at = w.doff + q;
        const uint32_t e = at >= 0 && at < w.staged ? w.s_dep[at] : __ldg(&w.dep_list[w.dfirst + at]);
        unsigned long long t0 = 0;
        const bool watched = (e & INTRA_DEP_WATCH) != 0, local = !(e & (INTRA_DEP_EXTERNAL | INTRA_DEP_WATCH));
        if ((local && e >= (uint32_t)w.task) || (watched && (int)(e & 0xFFu) >= w.n_watch)) {
            if (w.lane == 0) atomicOr(w.sticky, ST_BAD_RECORD);   // not an earlier TU, or no such watch slot: refused
            gave_up = true;
        } else if (local || watched) {
            uint64_t* bar = watched ? &w.s_wbar[e & 0xFFu] : &w.s_bar[e];
            for (unsigned polls = 0; !mbar_try_wait0(bar); polls++) {
                if (*w.s_abort) {
                    gave_up = true;
                    break;
                }
                const unsigned long long now = global_ns();
                if (polls == 0) t0 = now;
                if (now - t0 > WAIT_LIMIT_NS || polls >= SPIN_LIMIT) {
                    if (w.lane == 0) atomicOr(w.sticky, ST_TIMEOUT);
                    gave_up = true;
                    break;
                }
            }
        } else if ((e & ~INTRA_DEP_EXTERNAL) >= (uint32_t)w.n_itu) {
            if (w.lane == 0) atomicOr(w.sticky, ST_BAD_RECORD);
            gave_up = true;
        } else {
            cuda::atomic_ref<int32_t, cuda::thread_scope_device> f(w.itu_done[e & ~INTRA_DEP_EXTERNAL]);
            for (unsigned polls = 0; f.load(cuda::memory_order_relaxed) != w.epoch; polls++) {
                if ((polls & 255u) == 0) {   // the timer and the status words, every 256 polls
                    const unsigned long long now = global_ns();
                    if (polls == 0) t0 = now;
                    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> status(*w.sticky);
                    if (now - t0 > WAIT_LIMIT_NS || polls >= SPIN_LIMIT) {
                        if (w.lane == 0) atomicOr(w.sticky, ST_TIMEOUT);
                        gave_up = true;
                        break;
                    }
                    if (*w.s_abort || (status.load(cuda::memory_order_relaxed) & ST_TIMEOUT)) {
                        gave_up = true;
                        break;
                    }
                }
                __nanosleep(32);
            }
            if (!gave_up) cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
        }
        // the lanes may have seen a barrier, the abort word or the clock at different moments
        gave_up = __any_sync(0xffffffffu, gave_up);
    }
    // the warp barrier orders each lane's acquires before every lane's reads of the samples
    __syncwarp();
    return !gave_up;
}

__global__ void __launch_bounds__(IC_THREADS, IC_MIN_BLOCKS) k_intra_ctus(const __grid_constant__ SegTable st,
                                                                       int32_t* tickets, int total, uint32_t* sticky) {
    __shared__ __align__(16) uint8_t t_luma[IC_LH * IC_LP];
    __shared__ __align__(16) uint8_t t_chroma[2][IC_CH * IC_CP];
    __shared__ __align__(16) hevc_tu_t s_tu[IC_MAX_TUS];
    __shared__ __align__(16) int16_t s_res[IC_MAX_RES];
    __shared__ IntraWarpSmem ws[IC_WARPS];
    __shared__ uint64_t s_bar[IC_MAX_TUS];    // completion of the CTU's TUs, by task index
    __shared__ uint32_t s_itu_dep[IC_MAX_TUS];   // their dependency lists: (offset << 6) | count
    __shared__ uint32_t s_dep[IC_DEP_STAGE];     // the CTU's dependency entries
    __shared__ uint64_t s_wbar[IC_MAX_WATCH];    // completion of the watched TUs of other CTUs
    __shared__ uint32_t s_watch[IC_MAX_WATCH];   // their task indices in the picture
    __shared__ int s_ticket, s_pic, s_next;
    __shared__ IntraPic s_ipic;
    __shared__ volatile int s_abort;
    __shared__ uint32_t s_nb;
    const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    if (tid == 0) {
        // Each picture hands out its CTUs by ticket in wavefront order.  CTAs start at picture
        // blockIdx.x % n, so the pictures of a launch progress side by side; a picture whose
        // tickets are used up passes the CTA on.  There are as many CTAs as CTUs, so every
        // CTA finds one.
        int k = blockIdx.x % st.n, got = -1;
        for (int tries = 0; tries < st.n && got < 0; tries++) {
            const int n_k = (k + 1 < st.n ? st.s[k + 1].aux0 : total) - st.s[k].aux0;
            const int v = atomicAdd(&tickets[k], 1);
            if (v < n_k) got = v;
            else k = k + 1 == st.n ? 0 : k + 1;
        }
        // a wait of this launch (or an earlier one not yet read) gave up: the CTU could only
        // wait for work that will not come, so the CTA ends at once
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> status(*sticky);
        s_ticket = (status.load(cuda::memory_order_relaxed) & ST_TIMEOUT) ? -1 : got;
        s_pic = k;
        s_abort = 0;
        s_next = 0;
    }
    __syncthreads();
    if (s_ticket < 0) return;
    const int k = s_pic;
    const PicDesc& P = *st.s[k].pic;
    const int32_t epoch = st.s[k].aux1;
    const int idx = s_ticket;
    const int a = P.ictu_addr[idx], rx = a % P.wctb, ry = a / P.wctb;

    if (tid == 32) {
        s_ipic.rec = P.rec;
        s_ipic.off_cb = P.off_cb;
        s_ipic.off_cr = P.off_cr;
        s_ipic.width = P.width;
        s_ipic.height = P.height;
        s_ipic.log2_ctb = P.log2_ctb;
        s_ipic.pitch_y = P.pitch_y;
        s_ipic.pitch_c = P.pitch_c;
        s_ipic.intra_smoothing_disabled = P.intra_smoothing_disabled;
        s_ipic.strong_intra = P.strong_intra;
    }
    if (tid == 4) {  // which neighbour CTBs share this CTB's slice and tile
        const int sl = P.ctb_slice ? P.ctb_slice[a] : 0, ti = P.ctb_tile ? P.ctb_tile[a] : 0;
        auto same = [&](int nx, int ny) {
            if (nx < 0 || ny < 0 || nx >= P.wctb) return false;
            const int b = ny * P.wctb + nx;
            return (P.ctb_slice ? P.ctb_slice[b] : 0) == sl && (P.ctb_tile ? P.ctb_tile[b] : 0) == ti;
        };
        s_nb = (same(rx - 1, ry) ? NB_LEFT : 0u) | (same(rx - 1, ry - 1) ? NB_ABOVE_LEFT : 0u) |
               (same(rx, ry - 1) ? NB_ABOVE : 0u) | (same(rx + 1, ry - 1) ? NB_ABOVE_RIGHT : 0u);
    }

    // stage the CTU's tiles, TU records and residuals (packed in task order, one thread per
    // TU) in one round of asynchronous copies
    const int off = P.ictu_tu_off[idx], n_tu = P.ictu_tu_off[idx + 1] - off;
    for (int i = tid; i < n_tu; i += IC_THREADS) {
        cp_async16(&s_tu[i], &P.itu_rec[off + i]);
        mbar_init1(&s_bar[i]);
        s_itu_dep[i] = __ldg(&P.itu_dep[off + i]);
    }
    // the CTU's dependency entries are contiguous in task order
    const uint32_t dfirst = __ldg(&P.itu_dep[off]) >> 6, dlast_e = __ldg(&P.itu_dep[off + n_tu - 1]);
    const int n_dep = (int)((dlast_e >> 6) + (dlast_e & 63u)) - (int)dfirst;
    const int staged = max(0, min(n_dep, IC_DEP_STAGE));
    for (int q = tid; q < staged; q += IC_THREADS) s_dep[q] = __ldg(&P.dep_list[dfirst + q]);
    const uint32_t wd = __ldg(&P.ictu_watch[idx]);
    const int n_watch = min((int)(wd & 0xFFu), IC_MAX_WATCH);
    for (int q = tid; q < n_watch; q += IC_THREADS) {
        s_watch[q] = __ldg(&P.watch[(wd >> 8) + q]);
        mbar_init1(&s_wbar[q]);
    }
    stage_tile(P, 0, rx, ry, t_luma, tid);
    stage_tile(P, 1, rx, ry, t_chroma[0], tid);
    stage_tile(P, 2, rx, ry, t_chroma[1], tid);
    for (int i = tid; i < n_tu; i += IC_THREADS) {
        const int4 r = __ldg(&P.itu_res[off + i]);
        for (int c = 0; c < r.z; c++) cp_async16(s_res + r.y + 8 * c, P.resid + r.x + 8 * c);
    }
    cp_async_wait_all();
    __syncthreads();

    const int ctbl = 1 << P.log2_ctb;
    const uint32_t nb = s_nb;
    if (warp == IC_WATCHER) {
        // The watcher: one lane waits for the CTU's watched TUs of other CTUs in the order
        // their first dependent TU comes, polling each published completion through L2 and
        // sleeping between polls (the wait is bounded like every other), and arrives on the
        // TU's watch barrier when it sees it.  Its acquire, then that release arrival, order
        // the other CTU's samples before every read of a worker that waits on the barrier.
        if (lane == 0) {
            for (int j = 0; j < n_watch; j++) {
                if (s_watch[j] >= (uint32_t)P.n_itu) {   // no such TU: refused
                    atomicOr(sticky, ST_BAD_RECORD);
                    s_abort = 1;
                    break;
                }
                cuda::atomic_ref<int32_t, cuda::thread_scope_device> f(P.itu_done[s_watch[j]]);
                unsigned long long t0 = 0;
                unsigned nap = 32;
                bool gave_up = false;
                // relaxed polls (a GPU-scope acquire invalidates the SM's L1, which the
                // workers use), one acquire fence once the flag is seen
                for (unsigned polls = 0; f.load(cuda::memory_order_relaxed) != epoch; polls++) {
                    const unsigned long long now = global_ns();
                    if (polls == 0) t0 = now;
                    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> status(*sticky);
                    if (now - t0 > WAIT_LIMIT_NS || polls >= SPIN_LIMIT) {
                        atomicOr(sticky, ST_TIMEOUT);
                        gave_up = true;
                    } else if (s_abort || (status.load(cuda::memory_order_relaxed) & ST_TIMEOUT)) {
                        gave_up = true;
                    }
                    if (gave_up) break;
                    __nanosleep(nap);
                    nap = min(nap * 2, 256u);
                }
                if (gave_up) {
                    s_abort = 1;
                    break;
                }
                cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
                mbar_arrive(&s_wbar[j]);
            }
        }
        return;
    }
    for (;;) {
        int i = 0;
        if (lane == 0) i = s_abort ? n_tu : atomicAdd(&s_next, 1);
        i = __shfl_sync(0xffffffffu, i, 0);
        if (i >= n_tu) break;
        const hevc_tu_t tu = s_tu[i];
        const uint32_t dd = s_itu_dep[i];
        const int dcount = (int)(dd & 63u), doff = (int)(dd >> 6) - (int)dfirst;
        const IntraWait wc{s_dep, P.dep_list, s_bar, s_wbar, P.itu_done, sticky, &s_abort, (int)dfirst, doff, dcount,
                           staged, i, n_watch, P.n_itu, epoch, lane};
        auto wait = [&]() -> bool { return intra_wait(wc); };
        const int ctbc = tu.c_idx ? ctbl / 2 : ctbl;
        CtuTile tile;
        tile.t = tu.c_idx == 0 ? t_luma : t_chroma[tu.c_idx - 1];
        tile.pitch = tu.c_idx ? IC_CP : IC_LP;
        tile.x0 = rx * ctbc;
        tile.y0 = ry * ctbc;
        const int16_t* res = (tu.flags & HEVC_TU_CODED) ? s_res + tu.coeff_offset : nullptr;
        const bool done = tu.log2_size == 2   ? intra_tu4(s_ipic, tu, lane, tile, nb, res, wait)
                          : tu.log2_size == 3 ? intra_tu8(s_ipic, tu, lane, tile, nb, res, wait)
                          : tu.log2_size == 4 ? intra_tu16(s_ipic, tu, lane, ws[warp], tile, nb, res, wait)
                                              : intra_tu(s_ipic, tu, lane, ws[warp], tile, nb, res, wait);
        if (!done) {
            if (lane == 0) s_abort = 1;
            break;
        }
        // after the warp barrier, lane 0's release arrival and store order the warp's sample
        // writes (tile and picture) before the completion
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&s_bar[i]);
            if (tu.reserved[0] & ITU_PUBLISH) {
                cuda::atomic_ref<int32_t, cuda::thread_scope_device> g(P.itu_done[off + i]);
                g.store(epoch, cuda::memory_order_release);
            }
        }
    }
}

}  // namespace hevcgpu
