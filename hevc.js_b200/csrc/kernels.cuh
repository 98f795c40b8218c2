// kernels.cuh — the reconstruction kernels (sm_100a).
//
//   k_residual<LOG2>  dequant + inverse DST/DCT + add-and-clip of coded TUs
//                     (transform.cpp:293-394, coding_tree.cpp:371-396)
//   (motion compensation: mc.cuh; intra prediction: intra.cuh)
//   k_motion_grid     4x4 motion grid of the PUs (store_pu_motion's grid)
//   k_deblock<V>      Bs + decisions + luma/chroma filters of one edge direction
//                     (deblocking.cpp:50-614)
//   k_sao             band/edge offset from the deblocked picture into the DPB slot
//                     (sao.cpp:20-243)
//   k_picture_checksum  per-plane checksum of a frame (H.265 picture hash SEI, D.3.19)
#pragma once

#include "device_common.cuh"

namespace hevcgpu {

// ======================================================================================
// Inverse transform.  The N-point inverse DCT is computed by the even/odd recursion of
// the HEVC basis: out[k] = E[k] + O[k], out[N-1-k] = E[k] - O[k], with E the N/2-point
// inverse of the even inputs and O[k] the odd-input dot products.  The basis entries
// are integer cosines of pi*i*(2k+1)/64 (H.265 eq. 8-315); cos_mag lists the 33
// magnitudes for angles 0..pi/2 and every coefficient below is a compile-time constant.
// Integer sums are exact, so any summation order reproduces the reference's butterflies.
// ======================================================================================
__host__ __device__ constexpr int cos_mag(int m) {
    constexpr int t[33] = {64, 90, 90, 90, 89, 88, 87, 85, 83, 82, 80, 78, 75, 73, 70, 67, 64,
                           61, 57, 54, 50, 46, 43, 38, 36, 31, 25, 22, 18, 13, 9,  4,  0};
    return t[m];
}
__host__ __device__ constexpr int cos_entry(int m) {
    return (m & 127) <= 32 ? cos_mag(m & 127)
           : (m & 127) <= 64 ? -cos_mag(64 - (m & 127))
           : (m & 127) <= 96 ? -cos_mag((m & 127) - 64)
                             : cos_mag(128 - (m & 127));
}
// weight of input n in output k of the N-point inverse DCT
template <int N>
__host__ __device__ constexpr int dct_w(int n, int k) { return cos_entry(n * (32 / N) * (2 * k + 1)); }

template <int N>
__device__ __forceinline__ void idct_1d(const int* src, int* dst) {
    if constexpr (N == 2) {
        dst[0] = 64 * src[0] + 64 * src[1];
        dst[1] = 64 * src[0] - 64 * src[1];
    } else {
        int ev[N / 2], E[N / 2];
#pragma unroll
        for (int n = 0; n < N / 2; n++) ev[n] = src[2 * n];
        idct_1d<N / 2>(ev, E);
#pragma unroll
        for (int k = 0; k < N / 2; k++) {
            int o = 0;
#pragma unroll
            for (int n = 0; n < N / 2; n++) o += dct_w<N>(2 * n + 1, k) * src[2 * n + 1];
            dst[k] = E[k] + o;
            dst[N - 1 - k] = E[k] - o;
        }
    }
}

// DST-VII 4x4 (transform.cpp:22-43): out[k] = sum_n D[n][k] * src[n]
__device__ __forceinline__ void idst4_1d(const int* s, int* d) {
    d[0] = 29 * s[0] + 74 * s[1] + 84 * s[2] + 55 * s[3];
    d[1] = 55 * s[0] + 74 * s[1] - 29 * s[2] - 84 * s[3];
    d[2] = 74 * s[0] - 74 * s[2] + 74 * s[3];
    d[3] = 84 * s[0] - 74 * s[1] + 55 * s[2] - 29 * s[3];
}

template <int N>
__device__ __forceinline__ void inv_1d(const int* s, int* d, bool dst4) {
    if constexpr (N == 4) {
        if (dst4) { idst4_1d(s, d); return; }
    }
    idct_1d<N>(s, d);
}

// Dequantisation of one level (transform.cpp:360-365) with ms = m * levelScale[qP % 6]:
// the product, the shift by qP / 6 and the rounding shift in int64, narrowing to int
// (modulo 2^32), int16 clip.  |c * ms| <= 32768 * 255 * 72 fits an int.
__device__ __forceinline__ int16_t dequant1(int c, int ms, int qp_per, int bd_shift) {
    if (c == 0) return 0;
    long long v = (long long)(c * ms);
    v = v * (1ll << qp_per) + (1ll << (bd_shift - 1));
    v >>= bd_shift;
    return (int16_t)clip3(-32768, 32767, (int)(unsigned)(unsigned long long)v);
}

// Scaling factors m of row j of an N x N block (transform.cpp:320-358): matrixId is the
// plane plus 3 for a non-intra CU below 32x32, 0 or 3 at 32x32; a 4x4 block reads its
// list at j*4 + i, larger ones the 8x8 list at (j/r)*8 + i/r (r = N/8), and 16x16 and
// 32x32 blocks take the DC value (0 read as 16) at (0,0).  The lists sit 16-byte aligned,
// so a row is one 4- or 8-byte load.
template <int LOG2>
__device__ __forceinline__ void scaling_row(const hevc_scaling_t* S, int c_idx, bool intra, int j,
                                            int (&m)[1 << LOG2]) {
    constexpr int N = 1 << LOG2, SIZE_ID = LOG2 - 2;
    const int matrix = (SIZE_ID < 3 ? c_idx : 0) + (intra ? 0 : 3);
    const uint8_t* list = S->list[SIZE_ID][matrix];
    if constexpr (LOG2 == 2) {
        const uint32_t w = *reinterpret_cast<const uint32_t*>(list + 4 * j);
#pragma unroll
        for (int i = 0; i < 4; i++) m[i] = (w >> (8 * i)) & 255;
    } else {
        constexpr int R = N / 8;
        const uint2 w = *reinterpret_cast<const uint2*>(list + 8 * (j / R));
#pragma unroll
        for (int i = 0; i < N; i++) {
            const int k = i / R;
            m[i] = ((k < 4 ? w.x : w.y) >> (8 * (k & 3))) & 255;
        }
        if constexpr (LOG2 >= 4) {
            if (j == 0) {
                const int dc = S->dc[SIZE_ID - 2][matrix];
                m[0] = dc ? dc : 16;
            }
        }
    }
}

__constant__ int c_level_scale[6] = {40, 45, 51, 57, 64, 72};

// Residual kernel: N threads per TU (thread j owns column j in the first pass and row j
// in the second), 128 threads per CTA.  Coefficients are staged through shared memory;
// the intermediate has a padded row pitch (N + 2 int16) so that row reads by different
// threads hit distinct banks.
template <int LOG2>
__global__ void __launch_bounds__(128) k_residual(const __grid_constant__ SegTable st, int mode) {
    constexpr int N = 1 << LOG2;
    constexpr int TUS = 128 / N;
    constexpr int TP = N + 2;
    __shared__ __align__(16) int16_t s_coef[TUS][N * N];
    __shared__ int16_t s_tmp[TUS][N * TP];

    const int slot = threadIdx.x / N;
    const int j = threadIdx.x % N;
    const Seg& sg = st.s[find_seg(st, blockIdx.x)];
    const int item = (blockIdx.x - sg.block0) * TUS + slot;
    const bool live = item < sg.n_items;
    const PicDesc& P = *sg.pic;
    hevc_tu_t t = live ? P.tus[static_cast<const int32_t*>(sg.items)[item]] : hevc_tu_t{};
    const bool bypass = t.flags & (HEVC_TU_BYPASS | HEVC_TU_PCM);   // levels are the residual
    const bool tskip = (t.flags & HEVC_TU_TSKIP) && !bypass;
    const bool dst4 = (LOG2 == 2) && (t.flags & HEVC_TU_INTRA) && t.c_idx == 0;

    // load row j of the levels and dequantise it
    if (live) {
        const int16_t* src = P.coeffs + t.coeff_offset + j * N;
        int16_t v[N];
        if constexpr (N >= 8) {
#pragma unroll
            for (int q = 0; q < N / 8; q++) {
                int4 w = reinterpret_cast<const int4*>(src)[q];
                *reinterpret_cast<int4*>(&v[q * 8]) = w;
            }
        } else {
            int2 w = *reinterpret_cast<const int2*>(src);
            *reinterpret_cast<int2*>(&v[0]) = w;
        }
        if (!bypass) {
            const int scale = c_level_scale[t.qp % 6], qp_per = t.qp / 6, bd_shift = 8 + LOG2 - 5;
            if (P.scaling) {
                int m[N];
                scaling_row<LOG2>(P.scaling, t.c_idx, t.flags & HEVC_TU_INTRA, j, m);
#pragma unroll
                for (int i = 0; i < N; i++) v[i] = dequant1(v[i], m[i] * scale, qp_per, bd_shift);
            } else {
#pragma unroll
                for (int i = 0; i < N; i++) v[i] = dequant1(v[i], 16 * scale, qp_per, bd_shift);
            }
        }
#pragma unroll
        for (int i = 0; i < N; i++) s_coef[slot][j * N + i] = v[i];
    }
    __syncthreads();

    // first pass: column j, shift 7, int16 clip
    if (live && !tskip && !bypass) {
        int s[N], d[N];
#pragma unroll
        for (int n = 0; n < N; n++) s[n] = s_coef[slot][n * N + j];
        inv_1d<N>(s, d, dst4);
#pragma unroll
        for (int k = 0; k < N; k++) s_tmp[slot][k * TP + j] = (int16_t)clip3(-32768, 32767, (d[k] + 64) >> 7);
    }
    __syncthreads();
    if (!live) return;

    // second pass: row j, shift 12 (20 - BitDepth), int16 clip
    int r[N];
    if (bypass) {
#pragma unroll
        for (int k = 0; k < N; k++) r[k] = s_coef[slot][j * N + k];
    } else if (tskip) {
#pragma unroll
        for (int k = 0; k < N; k++) r[k] = (s_coef[slot][j * N + k] + 64) >> 7;
    } else {
        int s[N], d[N];
#pragma unroll
        for (int n = 0; n < N; n++) s[n] = s_tmp[slot][j * TP + n];
        inv_1d<N>(s, d, dst4);
#pragma unroll
        for (int k = 0; k < N; k++) r[k] = clip3(-32768, 32767, (d[k] + 2048) >> 12);
    }

    if (mode == RES_PICTURE && (t.flags & HEVC_TU_INTRA)) {
        // residual of an intra TU: the wavefront adds it to its prediction
        int16_t* dst = P.resid + t.coeff_offset + j * N;
#pragma unroll
        for (int k = 0; k < N; k++) dst[k] = (int16_t)r[k];
        return;
    }
    const uint8_t* pred;
    uint8_t* out;
    if (mode == RES_PACKED) {
        pred = P.rec + t.coeff_offset + j * N;
        out = P.dst + t.coeff_offset + j * N;
    } else {
        int pitch = t.c_idx ? P.pitch_c : P.pitch_y;
        int64_t base = t.c_idx == 0 ? 0 : (t.c_idx == 1 ? P.off_cb : P.off_cr);
        out = P.rec + base + (int64_t)(t.y + j) * pitch + t.x;
        pred = out;
    }
    // add the prediction row and clip (reconstruct_block)
    if constexpr (N >= 16) {
#pragma unroll
        for (int q = 0; q < N / 16; q++) {
            uint4 pv = reinterpret_cast<const uint4*>(pred)[q];
            const uint8_t* pb = reinterpret_cast<const uint8_t*>(&pv);
            uint4 ov;
            uint8_t* ob = reinterpret_cast<uint8_t*>(&ov);
#pragma unroll
            for (int i = 0; i < 16; i++) ob[i] = (uint8_t)clip_u8(pb[i] + r[q * 16 + i]);
            reinterpret_cast<uint4*>(out)[q] = ov;
        }
    } else if constexpr (N == 8) {
        uint2 pv = *reinterpret_cast<const uint2*>(pred);
        const uint8_t* pb = reinterpret_cast<const uint8_t*>(&pv);
        uint2 ov;
        uint8_t* ob = reinterpret_cast<uint8_t*>(&ov);
#pragma unroll
        for (int i = 0; i < 8; i++) ob[i] = (uint8_t)clip_u8(pb[i] + r[i]);
        *reinterpret_cast<uint2*>(out) = ov;
    } else {
        uint32_t pv = *reinterpret_cast<const uint32_t*>(pred);
        uint32_t ov = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) ov |= (uint32_t)clip_u8((int)((pv >> (8 * i)) & 0xFF) + r[i]) << (8 * i);
        *reinterpret_cast<uint32_t*>(out) = ov;
    }
}

// ======================================================================================
// Motion grid: one warp per PU writes its 4x4 entries (used by the Bs derivation).
// ======================================================================================
__global__ void k_motion_grid(const __grid_constant__ SegTable st) {
    const PicDesc& P = *st.s[blockIdx.y].pic;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
    if (warp >= P.num_pus) return;
    const hevc_pu_t pu = P.pus[warp];
    MotionEnt m;
    m.mv[0][0] = pu.mv[0][0]; m.mv[0][1] = pu.mv[0][1];
    m.mv[1][0] = pu.mv[1][0]; m.mv[1][1] = pu.mv[1][1];
    m.ref[0] = pu.ref_idx[0]; m.ref[1] = pu.ref_idx[1];
    m.pad = 0;
    const int bw = pu.w / 4, n = bw * (pu.h / 4), gw = P.width / 4;
    for (int e = lane; e < n; e += 32) {
        int gy = pu.y / 4 + e / bw, gx = pu.x / 4 + e % bw;
        P.mot[(int64_t)gy * gw + gx] = m;
    }
}

// ======================================================================================
// Deblocking.  One thread per 4-sample edge segment on the 8x8 grid; all segments of
// one direction are independent (each filters at most 3 samples either side and its
// decisions read 4, so neighbouring 8-spaced edges never touch the same samples), so
// the vertical pass and then the horizontal pass are each one launch.
// ======================================================================================
__constant__ uint8_t c_beta[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  6,  7,
                                   8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 20, 22, 24, 26, 28, 30, 32,
                                   34, 36, 38, 40, 42, 44, 46, 48, 50, 52, 54, 56, 58, 60, 62, 64};
__constant__ uint8_t c_tc[54] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1,  1,  1,  1,  1,  1,  1,  1,  1,
                                 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 8, 9, 10, 11, 13, 14, 16, 18, 20, 22, 24};
__constant__ uint8_t c_qpc[58] = {0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19,
                                  20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 29, 30, 31, 32, 33, 33, 34, 34, 35, 35,
                                  36, 36, 37, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51};

__device__ __forceinline__ int ref_poc_of(const PicDesc& P, const MotionEnt& m, int l) {
    const int r = l ? m.ref[1] : m.ref[0];
    return (r < 0 || r >= P.num_ref[l]) ? -999999 : P.ref_poc[l][r];
}
// |MV difference| >= 4 in either component, for list la of a and list lb of b (lists picked
// by value, so that the entries stay in registers)
__device__ __forceinline__ bool mv_far(const MotionEnt& a, int la, const MotionEnt& b, int lb) {
    const int ax = la ? a.mv[1][0] : a.mv[0][0], ay = la ? a.mv[1][1] : a.mv[0][1];
    const int bx = lb ? b.mv[1][0] : b.mv[0][0], by = lb ? b.mv[1][1] : b.mv[0][1];
    return abs(ax - bx) >= 4 || abs(ay - by) >= 4;
}

// derive_bs (deblocking.cpp:125-247), on the grid words and motion entries of the two sides
__device__ __forceinline__ int derive_bs(const PicDesc& P, uint32_t bp, uint32_t bq, const MotionEnt& mp,
                                         const MotionEnt& mq, int xp, int yp, int xq, int yq) {
    if ((bp | bq) & HEVC_BLK_INTRA) return 2;
    int tp = 1 << ((bp >> HEVC_BLK_TU_SHIFT) & 0xFF), tq = 1 << ((bq >> HEVC_BLK_TU_SHIFT) & 0xFF);
    bool tu_edge = (xp != xq) ? ((xq % tq == 0) || ((xp + 1) % tp == 0 && xp + 1 == xq))
                              : ((yq % tq == 0) || ((yp + 1) % tp == 0 && yp + 1 == yq));
    if (tu_edge && ((bp | bq) & HEVC_BLK_CBF)) return 1;
    int np = (mp.ref[0] >= 0) + (mp.ref[1] >= 0), nq = (mq.ref[0] >= 0) + (mq.ref[1] >= 0);
    if (np != nq) return 1;
    if (np == 1) {
        int lp = mp.ref[0] >= 0 ? 0 : 1, lq = mq.ref[0] >= 0 ? 0 : 1;
        if (ref_poc_of(P, mp, lp) != ref_poc_of(P, mq, lq)) return 1;
        return mv_far(mp, lp, mq, lq) ? 1 : 0;
    }
    if (np == 2) {
        int p0 = ref_poc_of(P, mp, 0), p1 = ref_poc_of(P, mp, 1), q0 = ref_poc_of(P, mq, 0), q1 = ref_poc_of(P, mq, 1);
        bool same = p0 == q0 && p1 == q1, swp = p0 == q1 && p1 == q0;
        if (!same && !swp) return 1;
        bool o1 = !mv_far(mp, 0, mq, 0) && !mv_far(mp, 1, mq, 1);
        bool o2 = !mv_far(mp, 0, mq, 1) && !mv_far(mp, 1, mq, 0);
        if (same && !swp) return o1 ? 0 : 1;
        if (!same && swp) return o2 ? 0 : 1;
        return (o1 || o2) ? 0 : 1;
    }
    return 0;
}

// Motion entry from its three words (the grid is 12-byte entries, 4-byte aligned).
__device__ __forceinline__ MotionEnt load_motion(const MotionEnt* g) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(g);
    const uint32_t a = w[0], b = w[1], c = w[2];
    MotionEnt m;
    m.mv[0][0] = (int16_t)(a & 0xFFFF);
    m.mv[0][1] = (int16_t)(a >> 16);
    m.mv[1][0] = (int16_t)(b & 0xFFFF);
    m.mv[1][1] = (int16_t)(b >> 16);
    m.ref[0] = (int8_t)(c & 0xFF);
    m.ref[1] = (int8_t)((c >> 8) & 0xFF);
    m.pad = 0;
    return m;
}

__device__ __forceinline__ const hevc_slice_t& slice_at(const PicDesc& P, int addr) {
    int s = P.ctb_slice ? P.ctb_slice[addr] : 0;
    return P.slices[s < P.num_slices ? s : 0];
}

// Filter one 4-sample luma segment held as p[line][i] (i = distance - 1 from the edge on
// the P side) and q[line][i]; returns the sample counts to write (per side, in
// nP/nQ) via the arrays themselves.
__device__ __forceinline__ void luma_segment(int (&p)[4][4], int (&q)[4][4], int beta, int tc, bool noP, bool noQ,
                                             int (&np)[4], int (&nq)[4]) {
    int dp0 = abs(p[0][2] - 2 * p[0][1] + p[0][0]), dp3 = abs(p[3][2] - 2 * p[3][1] + p[3][0]);
    int dq0 = abs(q[0][2] - 2 * q[0][1] + q[0][0]), dq3 = abs(q[3][2] - 2 * q[3][1] + q[3][0]);
    int dpq0 = dp0 + dq0, dpq3 = dp3 + dq3, dp = dp0 + dp3, dq = dq0 + dq3;
#pragma unroll
    for (int k = 0; k < 4; k++) np[k] = nq[k] = 0;
    if (dpq0 + dpq3 >= beta) return;
    bool strong = true;
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
        int k = kk * 3, dpq = kk ? dpq3 : dpq0;
        if (!(2 * dpq < (beta >> 2) && abs(p[k][3] - p[k][0]) + abs(q[k][0] - q[k][3]) < (beta >> 3) &&
              abs(p[k][0] - q[k][0]) < ((5 * tc + 1) >> 1)))
            strong = false;
    }
    int thr = (beta + (beta >> 1)) >> 3;
    bool dEp = dp < thr, dEq = dq < thr;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int P0 = p[k][0], P1 = p[k][1], P2 = p[k][2], P3 = p[k][3];
        int Q0 = q[k][0], Q1 = q[k][1], Q2 = q[k][2], Q3 = q[k][3];
        if (strong) {
            int t2 = 2 * tc;
            p[k][0] = clip3(P0 - t2, P0 + t2, (P2 + 2 * P1 + 2 * P0 + 2 * Q0 + Q1 + 4) >> 3);
            p[k][1] = clip3(P1 - t2, P1 + t2, (P2 + P1 + P0 + Q0 + 2) >> 2);
            p[k][2] = clip3(P2 - t2, P2 + t2, (2 * P3 + 3 * P2 + P1 + P0 + Q0 + 4) >> 3);
            q[k][0] = clip3(Q0 - t2, Q0 + t2, (P1 + 2 * P0 + 2 * Q0 + 2 * Q1 + Q2 + 4) >> 3);
            q[k][1] = clip3(Q1 - t2, Q1 + t2, (P0 + Q0 + Q1 + Q2 + 2) >> 2);
            q[k][2] = clip3(Q2 - t2, Q2 + t2, (P0 + Q0 + Q1 + 3 * Q2 + 2 * Q3 + 4) >> 3);
            np[k] = nq[k] = 3;
        } else {
            int delta = (9 * (Q0 - P0) - 3 * (Q1 - P1) + 8) >> 4;
            if (abs(delta) < tc * 10) {
                delta = clip3(-tc, tc, delta);
                p[k][0] = clip_u8(P0 + delta);
                q[k][0] = clip_u8(Q0 - delta);
                if (dEp) p[k][1] = clip_u8(P1 + clip3(-(tc >> 1), tc >> 1, (((P2 + P0 + 1) >> 1) - P1 + delta) >> 1));
                if (dEq) q[k][1] = clip_u8(Q1 + clip3(-(tc >> 1), tc >> 1, (((Q2 + Q0 + 1) >> 1) - Q1 - delta) >> 1));
                np[k] = dEp + 1;
                nq[k] = dEq + 1;
            }
        }
        if (noP) np[k] = 0;
        if (noQ) nq[k] = 0;
    }
}

#ifndef HEVCGPU_DEBLOCK_MIN_CTAS
#define HEVCGPU_DEBLOCK_MIN_CTAS 3   // CTAs of 256 threads per SM the register budget is sized for
#endif
template <bool VERT>
__global__ void __launch_bounds__(256, HEVCGPU_DEBLOCK_MIN_CTAS) k_deblock(const __grid_constant__ SegTable st) {
    const PicDesc& P = *st.s[blockIdx.y].pic;
    const int W = P.width, H = P.height, gw = W >> 2;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    // VERT: segments at x = 8i, y = 4j.  !VERT: x = 4i, y = 8j.
    const int nx = VERT ? (W + 7) >> 3 : W >> 2;
    const int x = VERT ? (tid % nx) * 8 : (tid % nx) * 4;
    const int y = VERT ? (tid / nx) * 4 : (tid / nx) * 8;
    if (y >= H || x >= W) return;
    if (VERT ? x == 0 : y == 0) return;
    const int xp = VERT ? x - 1 : x, yp = VERT ? y : y - 1;
    // Every load the segment may need is issued here, before any decision, so that the
    // segment waits for memory once: the grid words and motion entries of both sides, the
    // luma neighbourhood, and on the chroma grid the chroma neighbourhood.
    const uint32_t bq = P.blk[(int64_t)(y >> 2) * gw + (x >> 2)];
    const uint32_t bp = P.blk[(int64_t)(yp >> 2) * gw + (xp >> 2)];
    MotionEnt mp{}, mq{};
    if (P.mot) {
        mp = load_motion(P.mot + (int64_t)(yp >> 2) * gw + (xp >> 2));
        mq = load_motion(P.mot + (int64_t)(y >> 2) * gw + (x >> 2));
    }
    uint8_t* Y = P.rec;
    uint32_t wv[8];
    if (VERT) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint8_t* row = Y + (int64_t)(y + k) * P.pitch_y + x;
            wv[2 * k] = *reinterpret_cast<const uint32_t*>(row - 4);
            wv[2 * k + 1] = *reinterpret_cast<const uint32_t*>(row);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            wv[3 - i] = *reinterpret_cast<const uint32_t*>(Y + (int64_t)(y - 1 - i) * P.pitch_y + x);
            wv[4 + i] = *reinterpret_cast<const uint32_t*>(Y + (int64_t)(y + i) * P.pitch_y + x);
        }
    }
    // chroma (4:2:0): the segment's half on the 8-sample chroma grid, two lines of p1 p0 q0 q1
    // per plane; vertical edges as the words at cx - 4 and cx, horizontal ones as the words
    // of rows cy - 2 .. cy + 1 at the 4-aligned column holding cx .. cx + 1
    const bool cgrid = (((VERT ? x : y) >> 1) & 7) == 0;
    const int cx = x >> 1, cy = y >> 1, pc = P.pitch_c;
    uint32_t cw[2][4];
    if (cgrid) {
#pragma unroll
        for (int ci = 0; ci < 2; ci++) {
            const uint8_t* Cp = P.rec + (ci == 0 ? P.off_cb : P.off_cr);
            if (VERT) {
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const uint8_t* row = Cp + (int64_t)(cy + k) * pc + cx;
                    cw[ci][2 * k] = *reinterpret_cast<const uint32_t*>(row - 4);
                    cw[ci][2 * k + 1] = *reinterpret_cast<const uint32_t*>(row);
                }
            } else {
#pragma unroll
                for (int r = 0; r < 4; r++)
                    cw[ci][r] = *reinterpret_cast<const uint32_t*>(Cp + (int64_t)(cy - 2 + r) * pc + (cx & ~3));
            }
        }
    }

    if (!(bq & (VERT ? HEVC_BLK_EDGE_V : HEVC_BLK_EDGE_H))) return;
    const int aq = (y >> P.log2_ctb) * P.wctb + (x >> P.log2_ctb);
    const hevc_slice_t& sq = slice_at(P, aq);
    if (sq.deblocking_disabled) return;
    if (P.tiles_check || P.slice_check) {
        const int ap = (yp >> P.log2_ctb) * P.wctb + (xp >> P.log2_ctb);
        if (P.tiles_check && P.ctb_tile && P.ctb_tile[aq] != P.ctb_tile[ap]) return;
        if (P.slice_check && P.ctb_slice && P.ctb_slice[aq] != P.ctb_slice[ap] && !sq.lf_across_slices) return;
    }
    const int bs = derive_bs(P, bp, bq, mp, mq, xp, yp, x, y);
    if (bs == 0) return;
    const int qpP = (int8_t)(bp >> HEVC_BLK_QP_SHIFT), qpQ = (int8_t)(bq >> HEVC_BLK_QP_SHIFT);
    const bool noP = (P.pcm_lf_disabled && (bp & HEVC_BLK_PCM)) || (bp & HEVC_BLK_BYPASS);
    const bool noQ = (P.pcm_lf_disabled && (bq & HEVC_BLK_PCM)) || (bq & HEVC_BLK_BYPASS);
    const int qpl = (qpQ + qpP + 1) >> 1;
    const int beta = c_beta[clip3(0, 51, qpl + 2 * sq.beta_offset_div2)];
    const int tc = c_tc[clip3(0, 53, qpl + 2 * (bs - 1) + 2 * sq.tc_offset_div2)];

    // ---- luma: the 8x4 (or 4x8) neighbourhood from its words
    int p[4][4], q[4][4];
    if (VERT) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                p[k][i] = (wv[2 * k] >> (8 * (3 - i))) & 0xFF;
                q[k][i] = (wv[2 * k + 1] >> (8 * i)) & 0xFF;
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                p[k][i] = (wv[3 - i] >> (8 * k)) & 0xFF;
                q[k][i] = (wv[4 + i] >> (8 * k)) & 0xFF;
            }
    }
    int np[4], nq[4];
    luma_segment(p, q, beta, tc, noP, noQ, np, nq);
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; k++) any |= (np[k] | nq[k]) != 0;
    if (any) {
        if (VERT) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                uint32_t a = wv[2 * k], b = wv[2 * k + 1];
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    if (i < np[k]) a = (a & ~(0xFFu << (8 * (3 - i)))) | ((uint32_t)p[k][i] << (8 * (3 - i)));
                    if (i < nq[k]) b = (b & ~(0xFFu << (8 * i))) | ((uint32_t)q[k][i] << (8 * i));
                }
                uint8_t* row = Y + (int64_t)(y + k) * P.pitch_y + x;
                *reinterpret_cast<uint32_t*>(row - 4) = a;
                *reinterpret_cast<uint32_t*>(row) = b;
            }
        } else {
#pragma unroll
            for (int i = 0; i < 3; i++) {
                uint32_t a = wv[3 - i], b = wv[4 + i];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    if (i < np[k]) a = (a & ~(0xFFu << (8 * k))) | ((uint32_t)p[k][i] << (8 * k));
                    if (i < nq[k]) b = (b & ~(0xFFu << (8 * k))) | ((uint32_t)q[k][i] << (8 * k));
                }
                *reinterpret_cast<uint32_t*>(Y + (int64_t)(y - 1 - i) * P.pitch_y + x) = a;
                *reinterpret_cast<uint32_t*>(Y + (int64_t)(y + i) * P.pitch_y + x) = b;
            }
        }
    }

    // ---- chroma: Bs 2 on the 8-sample chroma grid (deblocking.cpp:538-609)
    if (bs == 2 && cgrid) {
#pragma unroll
        for (int ci = 0; ci < 2; ci++) {
            const int off = ci == 0 ? P.cb_qp_offset : P.cr_qp_offset;
            const int qpc = c_qpc[clip3(0, 57, ((qpQ + qpP + 1) >> 1) + off)];
            const int tcc = c_tc[clip3(0, 53, qpc + 2 + 2 * sq.tc_offset_div2)];
            uint8_t* Cp = P.rec + (ci == 0 ? P.off_cb : P.off_cr);
#pragma unroll
            for (int k = 0; k < 2; k++) {
                // p1 p0 | q0 q1 of line k
                int p0, p1, q0, q1;
                if (VERT) {
                    p1 = (cw[ci][2 * k] >> 16) & 0xFF;
                    p0 = cw[ci][2 * k] >> 24;
                    q0 = cw[ci][2 * k + 1] & 0xFF;
                    q1 = (cw[ci][2 * k + 1] >> 8) & 0xFF;
                } else {
                    const int sh = 8 * ((cx & 3) + k);
                    p1 = (cw[ci][0] >> sh) & 0xFF;
                    p0 = (cw[ci][1] >> sh) & 0xFF;
                    q0 = (cw[ci][2] >> sh) & 0xFF;
                    q1 = (cw[ci][3] >> sh) & 0xFF;
                }
                const int delta = clip3(-tcc, tcc, ((((q0 - p0) * 4) + p1 - q1 + 4) >> 3));
                uint8_t* s0 = VERT ? Cp + (int64_t)(cy + k) * pc + cx : Cp + (int64_t)cy * pc + cx + k;
                const int stp = VERT ? 1 : pc;
                if (!noP) s0[-stp] = (uint8_t)clip_u8(p0 + delta);
                if (!noQ) s0[0] = (uint8_t)clip_u8(q0 - delta);
            }
        }
    }
}

// ======================================================================================
// SAO: one thread per 8 horizontal samples of one plane (a group never straddles a CTB:
// CTBs are at least 8 samples wide in every plane), reading the deblocked picture (rec)
// with 8-byte loads and writing the DPB slot (dst); groups without SAO are copied.
// ======================================================================================
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

// Bytes x+d .. x+d+7 of a row from its words at x-4, x, x+4, x+8 (d in -1..1).
__device__ __forceinline__ void shifted_pair(uint32_t wm, uint32_t w0, uint32_t w1, uint32_t w2, int d,
                                             uint32_t& s0, uint32_t& s1) {
    if (d > 0) {
        s0 = __funnelshift_r(w0, w1, 8);
        s1 = __funnelshift_r(w1, w2, 8);
    } else {
        s0 = __funnelshift_rc(wm, w0, 32 + 8 * d);
        s1 = __funnelshift_rc(w0, w1, 32 + 8 * d);
    }
}

// SAO arithmetic on 16-bit lanes: two samples per 32-bit word, biased so that no lane
// borrows from its neighbour.  For a word of 4 samples c (and neighbours a, b), the even
// samples go to lanes as lo16(c0) | c2 << 16 and the odd ones as c1 | c3 << 16.
__device__ __forceinline__ uint32_t lanes_even(uint32_t w) { return prmt(w, 0u, 0x4240u); }
__device__ __forceinline__ uint32_t lanes_odd(uint32_t w) { return prmt(w, 0u, 0x4341u); }
// Offset-table selector for two lanes holding indices 0..5: nibbles [i0, 5, i1, 5] pick
// table byte i and the zero byte 5 as the lane's upper half.
__device__ __forceinline__ uint32_t lane_sel(uint32_t idx) { return prmt(idx + 0x00500050u, 0u, 0x4420u); }
// c + table offset (bytes of the table are offset + 8), clipped to 0..255, in lanes biased
// by 256; the low byte of each lane is the result.
__device__ __forceinline__ uint32_t lane_apply(uint32_t c, uint32_t tlo, uint32_t thi, uint32_t idx) {
    const uint32_t r = c + prmt(tlo, thi, lane_sel(idx)) + 0x00F800F8u;
    return __vmins2(__vmaxs2(r, 0x01000100u), 0x01FF01FFu);
}
// Edge index 2 + sign(c - a) + sign(c - b) per lane.
__device__ __forceinline__ uint32_t lane_edge(uint32_t c, uint32_t a, uint32_t b) {
    const uint32_t sa = __vmins2(__vmaxs2(c + 0x01000100u - a, 0x00FF00FFu), 0x01010101u);
    const uint32_t sb = __vmins2(__vmaxs2(c + 0x01000100u - b, 0x00FF00FFu), 0x01010101u);
    return sa + sb - 0x01FE01FEu;
}
// Band index (c >> 3) - band_position per lane, or 4 outside the four bands (no
// wrap-around, sao.cpp:229-230): (c >> 3) + 256 - pos keeps lanes apart, its low byte is
// the difference mod 256, and an unsigned min with 4 maps everything else to 4.
__device__ __forceinline__ uint32_t lane_band(uint32_t c, uint32_t k256) {
    return __vminu2(((c >> 3) + k256) & 0x00FF00FFu, 0x00040004u);
}
__device__ __forceinline__ uint32_t lanes_join(uint32_t even, uint32_t odd) { return prmt(even, odd, 0x6240u); }

// SAO of one CTB and plane per group of threads (apply_sao, sao.cpp:20-243): grid
// (CTB, picture, z) with z = 0 for luma (256 threads) and z = 1 for both chroma planes
// (128 threads each).  A thread takes 8 samples of a row, rows strided over the CTB.  The
// CTB's parameters are read once; samples are classified and offset branch-free on
// 16-bit lanes (edge offset: signs by clamping biased differences; band offset: band
// index by an unsigned min), the offset picked with one prmt from the five offset bytes.
// Samples the reference leaves unchanged — neighbour outside the picture, across a slice
// or tile boundary that filtering may not cross, PCM with pcm_loop_filter_disabled,
// transquant bypass — get their deblocked value back.  Reads the deblocked buffer (rec),
// writes the DPB slot (dst), so no full-picture copy is made.
__global__ void __launch_bounds__(256) k_sao(const __grid_constant__ SegTable st) {
    const PicDesc& P = *st.s[blockIdx.y].pic;
    const int ctb = blockIdx.x;
    if (ctb >= P.wctb * P.hctb) return;
    const int ci = blockIdx.z == 0 ? 0 : 1 + (threadIdx.x >> 7);
    const int T = blockIdx.z == 0 ? 256 : 128;
    const int t = blockIdx.z == 0 ? threadIdx.x : (threadIdx.x & 127);
    const int sub = ci ? 2 : 1;
    const int log2c = P.log2_ctb - (sub - 1);
    const int cs = 1 << log2c;
    const int pw = P.width / sub, ph = P.height / sub;
    const int cx = (ctb % P.wctb) << log2c, cy = (ctb / P.wctb) << log2c;
    const int G = cs >> 3;                 // 8-sample groups per CTB row (2..8)
    const int x = cx + (t % G) * 8;
    const int rstep = T / G;
    const int pitch = ci ? P.pitch_c : P.pitch_y;
    const int64_t base = ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr);
    const uint8_t* S = P.rec + base;
    uint8_t* D = P.dst + base;
    if (x >= pw) return;
    const int n = min(8, pw - x);          // 8, or 4 at the end of a row
    const int ymax = min(cy + cs, ph);

    const int type = P.sao_enabled ? P.sao[ctb].type[ci] : 0;
    if (type == 0) {
        for (int y = cy + t / G; y < ymax; y += rstep) {
            const int64_t at = (int64_t)y * pitch + x;
            const uint2 c8 = __ldg(reinterpret_cast<const uint2*>(S + at));
            if (n == 8) *reinterpret_cast<uint2*>(D + at) = c8;
            else *reinterpret_cast<uint32_t*>(D + at) = c8.x;
        }
        return;
    }
    const hevc_sao_t& sp = P.sao[ctb];
    // offset table: byte k = offset k + 8 (k = 0..4), byte 5 = 0 (the lanes' upper halves)
    uint32_t tlo = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) tlo |= (uint32_t)(uint8_t)(sp.offset[ci][k] + 8) << (8 * k);
    const uint32_t thi = type == 2 ? (uint32_t)(uint8_t)(sp.offset[ci][4] + 8) : 8u;
    const int cl = sp.eo_class[ci];
    const int dx = type == 2 ? (cl == 1 ? 0 : (cl == 3 ? 1 : -1)) : 0;   // a at (x+dx, y+dy), b opposite
    const int dy = type == 2 ? (cl == 0 ? 0 : -1) : 0;
    const uint32_t k256 = (uint32_t)(256 - sp.band_pos[ci]) * 0x00010001u;
    const bool check_slices = type == 2 && (P.slice_check || P.tiles_check);

    for (int y = cy + t / G; y < ymax; y += rstep) {
        const int64_t at = (int64_t)y * pitch + x;
        const uint2 c8 = __ldg(reinterpret_cast<const uint2*>(S + at));
        uint32_t o0 = c8.x, o1 = c8.y;
        bool apply = true;
        if (type == 2) {
            apply = y + dy >= 0 && y - dy < ph;
            if (apply) {
                uint32_t nw[2][2];
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int yy = y + (k ? -dy : dy);
                    const uint8_t* row = S + (int64_t)yy * pitch + x;
                    const uint2 m = yy == y ? c8 : __ldg(reinterpret_cast<const uint2*>(row));
                    const uint32_t wm = x >= 4 ? __ldg(reinterpret_cast<const uint32_t*>(row) - 1) : 0u;
                    const uint32_t w2 = x + 8 < pw ? __ldg(reinterpret_cast<const uint32_t*>(row) + 2) : 0u;
                    shifted_pair(wm, m.x, m.y, w2, k ? -dx : dx, nw[k][0], nw[k][1]);
                }
                o0 = lanes_join(lane_apply(lanes_even(c8.x), tlo, thi,
                                           lane_edge(lanes_even(c8.x), lanes_even(nw[0][0]), lanes_even(nw[1][0]))),
                                lane_apply(lanes_odd(c8.x), tlo, thi,
                                           lane_edge(lanes_odd(c8.x), lanes_odd(nw[0][0]), lanes_odd(nw[1][0]))));
                o1 = lanes_join(lane_apply(lanes_even(c8.y), tlo, thi,
                                           lane_edge(lanes_even(c8.y), lanes_even(nw[0][1]), lanes_even(nw[1][1]))),
                                lane_apply(lanes_odd(c8.y), tlo, thi,
                                           lane_edge(lanes_odd(c8.y), lanes_odd(nw[0][1]), lanes_odd(nw[1][1]))));
            }
        } else {
            o0 = lanes_join(lane_apply(lanes_even(c8.x), tlo, thi, lane_band(lanes_even(c8.x), k256)),
                            lane_apply(lanes_odd(c8.x), tlo, thi, lane_band(lanes_odd(c8.x), k256)));
            o1 = lanes_join(lane_apply(lanes_even(c8.y), tlo, thi, lane_band(lanes_even(c8.y), k256)),
                            lane_apply(lanes_odd(c8.y), tlo, thi, lane_band(lanes_odd(c8.y), k256)));
        }
        if (apply) {
            // samples that keep their deblocked value
            uint32_t keep = 0;
            if (dx != 0) {
                if (x == 0) keep |= 1u;
                if (x + n >= pw) keep |= 1u << (n - 1);
            }
            if (P.pcm_bypass_any || check_slices) {
                const int gw = P.width >> 2;
                for (int i = 0; i < n; i++) {
                    const int xs = x + i;
                    if (P.pcm_bypass_any) {
                        const uint32_t b = P.blk[(int64_t)((y * sub) >> 2) * gw + ((xs * sub) >> 2)];
                        if ((P.pcm_lf_disabled && (b & HEVC_BLK_PCM)) || (b & HEVC_BLK_BYPASS)) {
                            keep |= 1u << i;
                            continue;
                        }
                    }
                    if (!check_slices) continue;
                    const int cur = ((y * sub) >> P.log2_ctb) * P.wctb + ((xs * sub) >> P.log2_ctb);
                    for (int nk = 0; nk < 2; nk++) {
                        const int nx = xs + (nk ? -dx : dx), ny = y + (nk ? -dy : dy);
                        if (nx < 0 || nx >= pw) continue;   // kept above
                        const int na = ((ny * sub) >> P.log2_ctb) * P.wctb + ((nx * sub) >> P.log2_ctb);
                        const int sc = P.ctb_slice ? P.ctb_slice[cur] : 0, sn = P.ctb_slice ? P.ctb_slice[na] : 0;
                        if ((sc != sn && !slice_at(P, sn < sc ? cur : na).lf_across_slices) ||
                            (P.tiles_check && P.ctb_tile && P.ctb_tile[cur] != P.ctb_tile[na])) {
                            keep |= 1u << i;
                            break;
                        }
                    }
                }
            }
            if (keep) {
                uint32_t m0 = 0, m1 = 0;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    m0 |= ((keep >> i) & 1u) * (0xFFu << (8 * i));
                    m1 |= ((keep >> (i + 4)) & 1u) * (0xFFu << (8 * i));
                }
                o0 = (c8.x & m0) | (o0 & ~m0);
                o1 = (c8.y & m1) | (o1 & ~m1);
            }
        } else {
            o0 = c8.x;
            o1 = c8.y;
        }
        if (n == 8) *reinterpret_cast<uint2*>(D + at) = make_uint2(o0, o1);
        else *reinterpret_cast<uint32_t*>(D + at) = o0;
    }
}

// Frame output: the conformance window of a slot's three planes widened to 16-bit
// samples (the HEVCFrame planes of hevc_decoder_get_frame).  Plane p covers rows
// [0, h[p]) of its window; each thread writes 8 samples (one 16-byte store) of a staged
// row whose pitch is the window width rounded up to 8 samples, so every store is aligned;
// the bytes are read one by one (the window may start on any even column).
// The checksum of the H.265 decoded picture hash SEI (Rec. ITU-T H.265 D.3.19) of each
// plane of a frame, for 8-bit samples: the sum modulo 2^32 of sample ^ xorMask over the
// plane, xorMask = (x & 0xFF) ^ (y & 0xFF) ^ (x >> 8) ^ (y >> 8).  A sum, so the planes'
// rows are shared out over the CTAs (grid.y = plane) and the partial sums added atomically
// (32-bit wrap-around is the modulo).
struct ChecksumArgs {
    const uint8_t* src[3];
    int32_t pitch[3], w[3], h[3];
    uint32_t* out;   // three words, zero before the launch
};
__global__ void __launch_bounds__(256) k_picture_checksum(const __grid_constant__ ChecksumArgs a) {
    const int p = blockIdx.y;
    const int w = a.w[p], h = a.h[p];
    uint32_t sum = 0;
    for (int y = blockIdx.x; y < h; y += gridDim.x) {
        const uint8_t* row = a.src[p] + (int64_t)y * a.pitch[p];
        const uint32_t ym = (uint32_t)(y & 0xFF) ^ (uint32_t)(y >> 8);
        for (int x = threadIdx.x; x < w; x += blockDim.x)
            sum += (uint32_t)row[x] ^ ym ^ (uint32_t)(x & 0xFF) ^ (uint32_t)(x >> 8);
    }
    sum = __reduce_add_sync(0xffffffffu, sum);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(&a.out[p], sum);
}

struct WidenArgs {
    const uint8_t* src[3];   // first sample of the window in each plane of the slot
    int32_t src_pitch[3];
    uint16_t* dst[3];        // staged planes
    int32_t w[3], h[3], vecs[3];   // window size; 8-sample vectors per staged row
    int64_t first[3];              // first vector index of each plane (first[0] = 0)
    int64_t total;
};

__global__ void __launch_bounds__(256) k_widen_frame(const __grid_constant__ WidenArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.total) return;
    const int p = i >= a.first[2] ? 2 : (i >= a.first[1] ? 1 : 0);
    const int64_t k = i - a.first[p];
    const int row = (int)(k / a.vecs[p]), x0 = (int)(k % a.vecs[p]) * 8;
    const uint8_t* s = a.src[p] + (int64_t)row * a.src_pitch[p];
    uint32_t v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int x = x0 + 2 * q;
        const uint32_t lo = x < a.w[p] ? s[x] : 0u, hi = x + 1 < a.w[p] ? s[x + 1] : 0u;
        v[q] = lo | (hi << 16);
    }
    *reinterpret_cast<uint4*>(a.dst[p] + (int64_t)row * a.vecs[p] * 8 + x0) = make_uint4(v[0], v[1], v[2], v[3]);
}

}  // namespace hevcgpu
