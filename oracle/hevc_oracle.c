/*
 * hevc_oracle.c — CPU restatement of the hevc.js reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU back end is compared with;
 * nothing in the product links or calls it.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg use it.
 *
 * Each function restates one reference function of privaloops/hevc.js (cited by
 * path:line) on the record layouts of include/hevcgpu.h, including the reference's
 * deviations from the H.265 text (listed where they occur).  It is pinned against the
 * reference compiled from its own sources (oracle/_ref, built by oracle/Makefile) on
 * seeded inputs, and against the golden digests under tests/golden/.
 *
 * Planes are 8-bit I420, tightly packed.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/hevcgpu.h"

#define CLIP3(lo, hi, v) ((v) < (lo) ? (lo) : ((v) > (hi) ? (hi) : (v)))

typedef struct {
    uint8_t* p[3];
    int w[3], h[3];
} planes_t;

static void planes_of(uint8_t* base, int W, int H, planes_t* pl) {
    pl->w[0] = W; pl->h[0] = H;
    pl->w[1] = pl->w[2] = W / 2;
    pl->h[1] = pl->h[2] = H / 2;
    pl->p[0] = base;
    pl->p[1] = base + (size_t)W * H;
    pl->p[2] = pl->p[1] + (size_t)(W / 2) * (H / 2);
}

/* ------------------------------------------------------------------------------------
 * Transform matrices.  The N-point HEVC inverse DCT basis is the 32-point one sampled
 * every 32/N rows; entry (i, j) of the 32-point matrix is the integer cosine of
 * pi*i*(2j+1)/64, whose 33 magnitudes for angles 0..pi/2 are listed here (same
 * integers as transform.cpp:151-184 and H.265 eq. 8-315).  The DST-VII basis is the
 * 4x4 of transform.cpp:31.
 * ---------------------------------------------------------------------------------- */
static const int kCos[33] = {64, 90, 90, 90, 89, 88, 87, 85, 83, 82, 80, 78, 75, 73, 70, 67, 64,
                             61, 57, 54, 50, 46, 43, 38, 36, 31, 25, 22, 18, 13, 9,  4,  0};
static const int kDst[4][4] = {{29, 55, 74, 84}, {74, 74, 0, -74}, {84, -29, -74, 55}, {55, -84, 74, -29}};

static int cos_entry(int m) {
    m &= 127;
    if (m <= 32) return kCos[m];
    if (m <= 64) return -kCos[64 - m];
    if (m <= 96) return -kCos[m - 64];
    return kCos[128 - m];
}

/* basis[n][k]: weight of input coefficient n in output sample k. */
static void basis(int n_pts, int dst, int out[32][32]) {
    for (int n = 0; n < n_pts; n++)
        for (int k = 0; k < n_pts; k++)
            out[n][k] = dst ? kDst[n][k] : cos_entry(n * (32 / n_pts) * (2 * k + 1));
}

/* Scaling factor m of coefficient (x, y): perform_dequant, transform.cpp:320-358.
 * Flat 16 without lists.  sizeId = log2 - 2; matrixId = plane + 3 for a non-intra CU
 * below 32x32, 0 / 3 (intra / not) at 32x32 (:330-336).  4x4 reads list[0][matrixId]
 * at y*4 + x; larger sizes read list[sizeId][matrixId % 6] at (y/r)*8 + x/r, r = N/8,
 * capped at 63 (:343-347), and 16x16 / 32x32 take dc[sizeId-2][matrixId % 6] at (0,0),
 * where a 0 reads as 16 (:350-353). */
static int scale_factor(const hevc_scaling_t* sl, int log2, int c_idx, int intra, int x, int y) {
    if (!sl) return 16;
    int n = 1 << log2, size_id = log2 - 2, matrix;
    if (size_id < 3) matrix = c_idx + (intra ? 0 : 3);
    else matrix = intra ? 0 : 3;
    if (size_id == 0) return sl->list[0][matrix][y * n + x];
    int ratio = n / 8 < 1 ? 1 : n / 8;
    int idx = (y / ratio) * 8 + (x / ratio);
    if (idx > 63) idx = 63;
    int m = sl->list[size_id][matrix % 6][idx];
    if ((size_id == 2 || size_id == 3) && x == 0 && y == 0) {
        m = sl->dc[size_id - 2][matrix % 6];
        if (m == 0) m = 16;
    }
    return m;
}

/* Dequantisation: perform_dequant, transform.cpp:293-368.  The reference forms the
 * product in int64, shifts, then narrows to int before the int16 clip
 * (static_cast<int> at :365); the narrowing is modulo 2^32 here too (it bites only
 * with scaling factors above 16). */
static void dequant(const int16_t* c, int n, int qp, int bit_depth, const hevc_scaling_t* sl, int c_idx,
                    int intra, int16_t* d) {
    static const int level_scale[6] = {40, 45, 51, 57, 64, 72};
    int log2 = n == 4 ? 2 : n == 8 ? 3 : n == 16 ? 4 : 5;
    int bd_shift = bit_depth + log2 - 5;
    int64_t add = bd_shift > 0 ? ((int64_t)1 << (bd_shift - 1)) : 0;
    int64_t scale = level_scale[qp % 6];
    for (int i = 0; i < n * n; i++) {
        if (c[i] == 0) { d[i] = 0; continue; }
        int64_t v = (int64_t)c[i] * scale_factor(sl, log2, c_idx, intra, i % n, i / n) * scale;
        v = v * ((int64_t)1 << (qp / 6)) + add;
        v >>= bd_shift;
        int32_t narrowed = (int32_t)(uint32_t)(uint64_t)v;
        d[i] = (int16_t)CLIP3(-32768, 32767, narrowed);
    }
}

/* Two-pass inverse transform: inverse_transform_2d, transform.cpp:240-287
 * (columns with shift 7, int16 clip, rows with shift 20 - BitDepth, int16 clip);
 * transform skip and DST selection as perform_transform_inverse, :374-394. */
static void inverse_transform(const int16_t* d, int n, int flags, int c_idx, int bit_depth,
                              int16_t* r) {
    if (flags & HEVC_TU_TSKIP) {
        int shift = 15 - bit_depth > 0 ? 15 - bit_depth : 0;
        int add = shift > 0 ? 1 << (shift - 1) : 0;
        for (int i = 0; i < n * n; i++) r[i] = (int16_t)((d[i] + add) >> shift);
        return;
    }
    int use_dst = (flags & HEVC_TU_INTRA) && c_idx == 0 && n == 4;
    int B[32][32];   /* per call: the checkers run on several host threads at once */
    basis(n, use_dst, B);
    int16_t tmp[32 * 32];
    int s2 = 20 - bit_depth;
    for (int j = 0; j < n; j++)
        for (int k = 0; k < n; k++) {
            int acc = 0;
            for (int m = 0; m < n; m++) acc += B[m][k] * d[m * n + j];
            tmp[k * n + j] = (int16_t)CLIP3(-32768, 32767, (acc + 64) >> 7);
        }
    for (int y = 0; y < n; y++)
        for (int k = 0; k < n; k++) {
            int acc = 0;
            for (int m = 0; m < n; m++) acc += B[m][k] * tmp[y * n + m];
            r[y * n + k] = (int16_t)CLIP3(-32768, 32767, (acc + (1 << (s2 - 1))) >> s2);
        }
}

/* Residual of one TU (levels -> residual), including the transquant-bypass copy of
 * coding_tree.cpp:1302-1304. */
static void tu_residual(const hevc_tu_t* t, const int16_t* levels, int bit_depth, const hevc_scaling_t* sl,
                        int16_t* res) {
    int n = 1 << t->log2_size;
    if (!(t->flags & HEVC_TU_CODED)) { memset(res, 0, sizeof(int16_t) * n * n); return; }
    if (t->flags & (HEVC_TU_BYPASS | HEVC_TU_PCM)) { memcpy(res, levels, sizeof(int16_t) * n * n); return; }
    int16_t d[32 * 32];
    dequant(levels, n, t->qp, bit_depth, sl, t->c_idx, (t->flags & HEVC_TU_INTRA) != 0, d);
    inverse_transform(d, n, t->flags, t->c_idx, bit_depth, res);
}

int oracle_residual_blocks_scaled(const hevc_scaling_t* sl, const hevc_tu_t* tus, int32_t num_tus,
                                  const int16_t* coeffs, const uint8_t* pred, uint8_t* out) {
    int16_t res[32 * 32];
    for (int t = 0; t < num_tus; t++) {
        const hevc_tu_t* tu = &tus[t];
        if (tu->log2_size < 2 || tu->log2_size > 5) return -1;
        int n = 1 << tu->log2_size;
        tu_residual(tu, coeffs + tu->coeff_offset, 8, sl, res);
        /* reconstruct_block, coding_tree.cpp:371-396 */
        for (int i = 0; i < n * n; i++) {
            int v = pred[tu->coeff_offset + i] + res[i];
            out[tu->coeff_offset + i] = (uint8_t)CLIP3(0, 255, v);
        }
    }
    return 0;
}

int oracle_residual_blocks(const hevc_tu_t* tus, int32_t num_tus, const int16_t* coeffs,
                           const uint8_t* pred, uint8_t* out) {
    return oracle_residual_blocks_scaled(NULL, tus, num_tus, coeffs, pred, out);
}

/* ------------------------------------------------------------------------------------
 * Inter prediction: interpolate_luma / interpolate_chroma (interpolation.cpp:45-209),
 * weighted_pred_default / weighted_pred_explicit (:215-300), perform_inter_prediction
 * (:306-411).  Reference samples outside the picture repeat the edge sample (refClamp,
 * :64-68).  8-bit: shift1 = 0, shift2 = 6, shift3 = 6.
 * ---------------------------------------------------------------------------------- */
static const int kLumaTaps[4][8] = {{0, 0, 0, 64, 0, 0, 0, 0},
                                    {-1, 4, -10, 58, 17, -5, 1, 0},
                                    {-1, 4, -11, 40, 40, -11, 4, -1},
                                    {0, 1, -5, 17, 58, -10, 4, -1}};
static const int kChromaTaps[8][4] = {{0, 64, 0, 0},     {-2, 58, 10, -2}, {-4, 54, 16, -2},
                                      {-6, 46, 28, -4},  {-4, 36, 36, -4}, {-4, 28, 46, -6},
                                      {-2, 16, 54, -4},  {-2, 10, 58, -2}};

static int ref_at(const uint8_t* p, int w, int h, int x, int y) {
    x = CLIP3(0, w - 1, x);
    y = CLIP3(0, h - 1, y);
    return p[(size_t)y * w + x];
}

/* One component, one list: the 14-bit intermediate prediction (int16). */
static void interp(const uint8_t* ref, int pw, int ph, int x_int, int y_int, int fx, int fy,
                   int bw, int bh, int ntaps, int16_t* dst) {
    const int* th = ntaps == 8 ? kLumaTaps[fx] : kChromaTaps[fx];
    const int* tv = ntaps == 8 ? kLumaTaps[fy] : kChromaTaps[fy];
    int half = ntaps / 2 - 1; /* 3 for luma, 1 for chroma */
    if (fx == 0 && fy == 0) {
        for (int y = 0; y < bh; y++)
            for (int x = 0; x < bw; x++)
                dst[y * bw + x] = (int16_t)(ref_at(ref, pw, ph, x_int + x, y_int + y) << 6);
        return;
    }
    if (fy == 0) {
        for (int y = 0; y < bh; y++)
            for (int x = 0; x < bw; x++) {
                int s = 0;
                for (int k = 0; k < ntaps; k++) s += th[k] * ref_at(ref, pw, ph, x_int + x + k - half, y_int + y);
                dst[y * bw + x] = (int16_t)s;
            }
        return;
    }
    if (fx == 0) {
        for (int y = 0; y < bh; y++)
            for (int x = 0; x < bw; x++) {
                int s = 0;
                for (int k = 0; k < ntaps; k++) s += tv[k] * ref_at(ref, pw, ph, x_int + x, y_int + y + k - half);
                dst[y * bw + x] = (int16_t)s;
            }
        return;
    }
    int16_t tmp[(64 + 7) * 64];
    int th_rows = bh + ntaps - 1;
    for (int y = 0; y < th_rows; y++)
        for (int x = 0; x < bw; x++) {
            int s = 0;
            for (int k = 0; k < ntaps; k++) s += th[k] * ref_at(ref, pw, ph, x_int + x + k - half, y_int + y - half);
            tmp[y * bw + x] = (int16_t)s;
        }
    for (int y = 0; y < bh; y++)
        for (int x = 0; x < bw; x++) {
            int s = 0;
            for (int k = 0; k < ntaps; k++) s += tv[k] * tmp[(y + k) * bw + x];
            dst[y * bw + x] = (int16_t)(s >> 6);
        }
}

static int pu_pred(const hevc_pic_params_t* pp, const hevc_pu_t* pu, const hevc_wp_t* wp_tab,
                   int num_wp, const uint8_t* const* refs, int num_refs, planes_t* out) {
    int W = pp->width, H = pp->height;
    int16_t pl[2][64 * 64];
    int use[2];
    const hevc_wp_t* wp = NULL;
    if (pu->wp >= 0) {
        if (pu->wp >= num_wp) return -1;
        wp = &wp_tab[pu->wp];
    }
    if (pu->w < 4 || pu->h < 4 || pu->w > 64 || pu->h > 64 || pu->x + pu->w > W || pu->y + pu->h > H)
        return -1;
    for (int ci = 0; ci < 3; ci++) {
        int sw = ci ? 2 : 1;
        int bw = pu->w / sw, bh = pu->h / sw;
        int pw = W / sw, ph = H / sw;
        for (int l = 0; l < 2; l++) {
            use[l] = pu->ref_idx[l] >= 0;
            if (!use[l]) continue;
            if (pu->ref_idx[l] >= pp->num_ref[l]) return -1;
            int slot = pp->ref_slot[l][pu->ref_idx[l]];
            if (slot < 0 || slot >= num_refs) return -1;
            planes_t rp;
            planes_of((uint8_t*)refs[slot], W, H, &rp);
            int mvx = pu->mv[l][0], mvy = pu->mv[l][1];
            if (ci == 0)
                interp(rp.p[0], pw, ph, pu->x + (mvx >> 2), pu->y + (mvy >> 2), mvx & 3, mvy & 3, bw, bh, 8, pl[l]);
            else
                interp(rp.p[ci], pw, ph, pu->x / 2 + (mvx >> 3), pu->y / 2 + (mvy >> 3), mvx & 7, mvy & 7, bw, bh, 4, pl[l]);
        }
        if (!use[0] && !use[1]) return -1;
        uint8_t* dst = out->p[ci];
        int ox = pu->x / sw, oy = pu->y / sw;
        for (int y = 0; y < bh; y++)
            for (int x = 0; x < bw; x++) {
                int i = y * bw + x, v;
                if (!wp) {
                    if (use[0] && use[1]) v = (pl[0][i] + pl[1][i] + 64) >> 7;
                    else v = ((use[0] ? pl[0][i] : pl[1][i]) + 32) >> 6;
                } else {
                    int lw = wp->log2wd[ci ? 1 : 0];
                    if (use[0] && use[1])
                        v = (pl[0][i] * wp->w[0][ci] + pl[1][i] * wp->w[1][ci] +
                             ((wp->o[0][ci] + wp->o[1][ci] + 1) << lw)) >> (lw + 1);
                    else {
                        int l = use[0] ? 0 : 1;
                        v = ((pl[l][i] * wp->w[l][ci] + (1 << (lw - 1))) >> lw) + wp->o[l][ci];
                    }
                }
                dst[(size_t)(oy + y) * out->w[ci] + ox + x] = (uint8_t)CLIP3(0, 255, v);
            }
    }
    return 0;
}

int oracle_inter_pred(const hevc_pic_params_t* pp, const hevc_pu_t* pus, int32_t num_pus,
                      const hevc_wp_t* wp, int32_t num_wp, const uint8_t* const* refs,
                      int32_t num_refs, uint8_t* out) {
    planes_t o;
    planes_of(out, pp->width, pp->height, &o);
    for (int i = 0; i < num_pus; i++)
        if (pu_pred(pp, &pus[i], wp, num_wp, refs, num_refs, &o)) return -1;
    return 0;
}

/* ------------------------------------------------------------------------------------
 * Intra prediction: perform_intra_prediction (intra_prediction.cpp:428-481) and its
 * helpers.  Availability (build_reference_samples, :44-211): a neighbouring sample is
 * usable when it lies in the picture and either in an earlier CTB (raster order) of
 * the same slice and tile, or in the current CTB at a 4x4-luma z-scan address below
 * that of the TU's top-left corner.
 * ---------------------------------------------------------------------------------- */
static const int kAngle[35] = {0,   0,   32,  26,  21,  17,  13,  9,  5,  2,  0,  -2,
                               -5,  -9,  -13, -17, -21, -26, -32, -26, -21, -17, -13, -9,
                               -5,  -2,  0,   2,   5,   9,   13,  17,  21,  26,  32};
static const int kInvAngle[35] = {0,    0,    256, 315, 390, 482,  630,  910,  1638, 4096, 0,   4096,
                                  1638, 910,  630, 482, 390, 315,  256,  315,  390,  482,  630, 910,
                                  1638, 4096, 0,   4096, 1638, 910, 630, 482,  390,  315,  256};

static uint32_t zorder(int bx, int by) {
    uint32_t z = 0;
    for (int i = 0; i < 8; i++) z |= (uint32_t)((bx >> i) & 1) << (2 * i) | (uint32_t)((by >> i) & 1) << (2 * i + 1);
    return z;
}

typedef struct {
    const hevc_picture_syntax_t* syn;
    int W, H, ctb, wctb;
} intra_env_t;

static int ctb_slice(const intra_env_t* e, int a) { return e->syn->ctb_slice ? e->syn->ctb_slice[a] : 0; }
static int ctb_tile(const intra_env_t* e, int a) {
    return (e->syn->params.tiles_enabled && e->syn->ctb_tile) ? e->syn->ctb_tile[a] : 0;
}

static void intra_tu(const intra_env_t* e, const hevc_tu_t* t, const int16_t* res, planes_t* pic) {
    int ci = t->c_idx, sub = ci ? 2 : 1;
    int n = 1 << t->log2_size;
    int pw = e->W / sub, ph = e->H / sub;
    int xc = t->x, yc = t->y;          /* component coordinates                    */
    int x0 = xc * sub, y0 = yc * sub;  /* luma position the reference is called with */
    int ctb_c = e->ctb / sub;
    int cur_cx = xc / ctb_c, cur_cy = yc / ctb_c;
    int cur_addr = cur_cy * e->wctb + cur_cx;
    int ox = cur_cx * e->ctb, oy = cur_cy * e->ctb;
    uint32_t cur_z = zorder((x0 - ox) / 4, (y0 - oy) / 4);
    const uint8_t* P = pic->p[ci];

    /* samples[0..4n]: bottom-left upward, corner at 2n, then top row to the right */
    int total = 4 * n + 1;
    int s[4 * 32 + 1], av[4 * 32 + 1];
    for (int i = 0; i < total; i++) {
        int rx, ry;
        if (i < 2 * n) { rx = xc - 1; ry = yc + 2 * n - 1 - i; }
        else if (i == 2 * n) { rx = xc - 1; ry = yc - 1; }
        else { rx = xc + (i - 2 * n - 1); ry = yc - 1; }
        int ok = 0;
        if (rx >= 0 && ry >= 0 && rx < pw && ry < ph) {
            int cx = rx / ctb_c, cy = ry / ctb_c;
            if (cx != cur_cx || cy != cur_cy) {
                int a = cy * e->wctb + cx;
                ok = a < cur_addr && ctb_slice(e, a) == ctb_slice(e, cur_addr) &&
                     ctb_tile(e, a) == ctb_tile(e, cur_addr);
            } else {
                ok = zorder((rx * sub - ox) / 4, (ry * sub - oy) / 4) < cur_z;
            }
        }
        av[i] = ok;
        s[i] = ok ? P[(size_t)ry * pw + rx] : 0;
    }
    int first = -1;
    for (int i = 0; i < total; i++) if (av[i]) { first = i; break; }
    if (first < 0) {
        for (int i = 0; i < total; i++) s[i] = 128;
    } else {
        for (int i = 0; i < first; i++) s[i] = s[first];
        for (int i = first + 1; i < total; i++) if (!av[i]) s[i] = s[i - 1];
    }
    /* top[0] = corner, top[1..2n] = row; left[0] = corner, left[1..2n] = column down */
    int top[2 * 32 + 1], left[2 * 32 + 1];
    top[0] = left[0] = s[2 * n];
    for (int i = 0; i < 2 * n; i++) { top[1 + i] = s[2 * n + 1 + i]; left[1 + i] = s[2 * n - 1 - i]; }

    int mode = t->intra_mode;
    /* filtering (:443-471): luma only for 4:2:0 */
    int filt = 0;
    if (!e->syn->params.intra_smoothing_disabled && ci == 0 && mode != 1 && n != 4) {
        int d = abs(mode - 26) < abs(mode - 10) ? abs(mode - 26) : abs(mode - 10);
        int thr = n == 8 ? 7 : n == 16 ? 1 : 0;
        filt = d > thr;
    }
    if (filt) {
        int bilinear = 0;
        if (e->syn->params.strong_intra_smoothing && n == 32) {
            int thr = 1 << (8 - 5);
            bilinear = abs(top[0] + top[2 * n] - 2 * top[n]) < thr && abs(left[0] + left[2 * n] - 2 * left[n]) < thr;
        }
        int nt[2 * 32 + 1], nl[2 * 32 + 1];
        if (bilinear) {
            for (int i = 1; i < 2 * n; i++) {
                nt[i] = ((2 * n - i) * top[0] + i * top[2 * n] + n) / (2 * n);
                nl[i] = ((2 * n - i) * left[0] + i * left[2 * n] + n) / (2 * n);
            }
            nt[0] = top[0]; nl[0] = left[0];
        } else {
            for (int i = 1; i < 2 * n; i++) {
                nt[i] = (top[i - 1] + 2 * top[i] + top[i + 1] + 2) >> 2;
                nl[i] = (left[i - 1] + 2 * left[i] + left[i + 1] + 2) >> 2;
            }
            nt[0] = nl[0] = (left[1] + 2 * top[0] + top[1] + 2) >> 2;
        }
        nt[2 * n] = top[2 * n]; nl[2 * n] = left[2 * n];
        memcpy(top, nt, sizeof(int) * (2 * n + 1));
        memcpy(left, nl, sizeof(int) * (2 * n + 1));
    }

    int pred[32 * 32];
    int log2 = t->log2_size;
    if (mode == 0) { /* predict_planar :263-289 */
        for (int y = 0; y < n; y++)
            for (int x = 0; x < n; x++)
                pred[y * n + x] = ((n - 1 - x) * left[y + 1] + (x + 1) * top[n + 1] + (n - 1 - y) * top[x + 1] +
                                   (y + 1) * left[n + 1] + n) >> (log2 + 1);
    } else if (mode == 1) { /* predict_dc :295-317 */
        int sum = 0;
        for (int i = 1; i <= n; i++) sum += top[i] + left[i];
        int dc = (sum + n) >> (log2 + 1);
        for (int i = 0; i < n * n; i++) pred[i] = dc;
        if (ci == 0 && n < 32) {
            pred[0] = (top[1] + left[1] + 2 * dc + 2) >> 2;
            for (int x = 1; x < n; x++) pred[x] = (top[x + 1] + 3 * dc + 2) >> 2;
            for (int y = 1; y < n; y++) pred[y * n] = (left[y + 1] + 3 * dc + 2) >> 2;
        }
    } else { /* predict_angular :323-422 */
        int ang = kAngle[mode];
        int vert = mode >= 18;
        const int* main_ref = vert ? top : left;
        const int* side_ref = vert ? left : top;
        int ext[3 * 64 + 2];
        int off = 64;
        for (int i = 0; i <= 2 * n; i++) ext[off + i] = main_ref[i];
        if (ang < 0) {
            int neg = (-(n * ang) + 31) >> 5;
            for (int i = 1; i <= neg; i++) {
                int si = (i * kInvAngle[mode] + 128) >> 8;
                if (si > 2 * n) si = 2 * n;
                ext[off - i] = side_ref[si];
            }
        }
        const int* ref = ext + off;
        for (int y = 0; y < n; y++)
            for (int x = 0; x < n; x++) {
                int pos = vert ? y : x, lane = vert ? x : y;
                int idx = ((pos + 1) * ang) >> 5, fr = ((pos + 1) * ang) & 31;
                int ri = lane + 1 + idx;
                pred[y * n + x] = fr ? ((32 - fr) * ref[ri] + fr * ref[ri + 1] + 16) >> 5 : ref[ri];
            }
        if (ci == 0 && n < 32) {
            if (mode == 26)
                for (int y = 0; y < n; y++) pred[y * n] = CLIP3(0, 255, pred[y * n] + ((left[y + 1] - left[0]) >> 1));
            else if (mode == 10)
                for (int x = 0; x < n; x++) pred[x] = CLIP3(0, 255, pred[x] + ((top[x + 1] - top[0]) >> 1));
        }
    }
    /* a PCM block's samples are its levels (coding_tree.cpp:1425-1469): no prediction */
    int pcm = (t->flags & HEVC_TU_PCM) != 0;
    uint8_t* D = pic->p[ci];
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
            if (xc + x >= pw || yc + y >= ph) continue;
            int v = (pcm ? 0 : (int16_t)pred[y * n + x]) + (res ? res[y * n + x] : 0);
            D[(size_t)(yc + y) * pw + xc + x] = (uint8_t)CLIP3(0, 255, v);
        }
}

static void inter_residuals(const hevc_picture_syntax_t* syn, planes_t* pic) {
    int16_t res[32 * 32];
    for (int i = 0; i < syn->num_tus; i++) {
        const hevc_tu_t* t = &syn->tus[i];
        if ((t->flags & HEVC_TU_INTRA) || !(t->flags & HEVC_TU_CODED)) continue;
        int n = 1 << t->log2_size, ci = t->c_idx;
        tu_residual(t, syn->coeffs + t->coeff_offset, 8, syn->scaling, res);
        for (int y = 0; y < n; y++)
            for (int x = 0; x < n; x++) {
                if (t->x + x >= pic->w[ci] || t->y + y >= pic->h[ci]) continue;
                uint8_t* s = &pic->p[ci][(size_t)(t->y + y) * pic->w[ci] + t->x + x];
                *s = (uint8_t)CLIP3(0, 255, *s + res[y * n + x]);
            }
    }
}

static void intra_pass(const hevc_picture_syntax_t* syn, planes_t* pic) {
    intra_env_t e;
    e.syn = syn;
    e.W = syn->params.width;
    e.H = syn->params.height;
    e.ctb = 1 << syn->params.log2_ctb;
    e.wctb = (e.W + e.ctb - 1) / e.ctb;
    int16_t res[32 * 32];
    for (int i = 0; i < syn->num_tus; i++) {
        const hevc_tu_t* t = &syn->tus[i];
        if (!(t->flags & HEVC_TU_INTRA)) continue;
        const int16_t* r = NULL;
        if (t->flags & HEVC_TU_CODED) {
            tu_residual(t, syn->coeffs + t->coeff_offset, 8, syn->scaling, res);
            r = res;
        }
        intra_tu(&e, t, r, pic);
    }
}

int oracle_intra_recon(const hevc_picture_syntax_t* syn, const uint8_t* in, uint8_t* out) {
    size_t sz = (size_t)syn->params.width * syn->params.height * 3 / 2;
    if (out != in) memcpy(out, in, sz);
    planes_t pic;
    planes_of(out, syn->params.width, syn->params.height, &pic);
    intra_pass(syn, &pic);
    return 0;
}

/* ------------------------------------------------------------------------------------
 * Deblocking: apply_deblocking (deblocking.cpp:357-614) with derive_bs (:125-247),
 * is_boundary_excluded (:50-120), the luma decisions (:434-493, :266) and filters
 * (:279-352).  All vertical edges of the picture, then all horizontal edges.
 * ---------------------------------------------------------------------------------- */
static const int kBeta[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  6,  7,
                              8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 20, 22, 24, 26, 28, 30, 32,
                              34, 36, 38, 40, 42, 44, 46, 48, 50, 52, 54, 56, 58, 60, 62, 64};
static const int kTc[54] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1,  1,  1,  1,  1,  1,  1,  1,  1,
                            2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 8, 9, 10, 11, 13, 14, 16, 18, 20, 22, 24};
static const int kQpc[58] = {0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19,
                             20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 29, 30, 31, 32, 33, 33, 34, 34, 35, 35,
                             36, 36, 37, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51};

typedef struct { int16_t mv[2][2]; int8_t ref[2]; } mot_t;

typedef struct {
    const hevc_picture_syntax_t* syn;
    int W, H, gw, ctb, wctb;
    mot_t* mot;
} dbk_env_t;

static uint32_t blk_at(const dbk_env_t* e, int x, int y) { return e->syn->blk[(size_t)(y / 4) * e->gw + x / 4]; }
static const hevc_slice_t* slice_of(const dbk_env_t* e, int addr) {
    int s = e->syn->ctb_slice ? e->syn->ctb_slice[addr] : 0;
    if (s >= e->syn->num_slices) s = 0;
    return &e->syn->slices[s];
}
static int ref_poc(const dbk_env_t* e, const mot_t* m, int l) {
    int r = m->ref[l];
    if (r < 0 || r >= e->syn->params.num_ref[l]) return -999999;
    return e->syn->params.ref_poc[l][r];
}
static int mv_far(const int16_t* a, const int16_t* b) { return abs(a[0] - b[0]) >= 4 || abs(a[1] - b[1]) >= 4; }

static int derive_bs(const dbk_env_t* e, int xp, int yp, int xq, int yq) {
    uint32_t bp = blk_at(e, xp, yp), bq = blk_at(e, xq, yq);
    if ((bp | bq) & HEVC_BLK_INTRA) return 2;
    int tp = 1 << ((bp >> HEVC_BLK_TU_SHIFT) & 0xFF), tq = 1 << ((bq >> HEVC_BLK_TU_SHIFT) & 0xFF);
    /* the reference's TU-edge test, deblocking.cpp:159-166 */
    int tu_edge = (xp != xq) ? ((xq % tq == 0) || ((xp + 1) % tp == 0 && xp + 1 == xq))
                             : ((yq % tq == 0) || ((yp + 1) % tp == 0 && yp + 1 == yq));
    if (tu_edge && ((bp | bq) & HEVC_BLK_CBF)) return 1;
    const mot_t* mp = &e->mot[(size_t)(yp / 4) * e->gw + xp / 4];
    const mot_t* mq = &e->mot[(size_t)(yq / 4) * e->gw + xq / 4];
    int np = (mp->ref[0] >= 0) + (mp->ref[1] >= 0), nq = (mq->ref[0] >= 0) + (mq->ref[1] >= 0);
    if (np != nq) return 1;
    if (np == 1) {
        int lp = mp->ref[0] >= 0 ? 0 : 1, lq = mq->ref[0] >= 0 ? 0 : 1;
        if (ref_poc(e, mp, lp) != ref_poc(e, mq, lq)) return 1;
        return mv_far(mp->mv[lp], mq->mv[lq]);
    }
    if (np == 2) {
        int p0 = ref_poc(e, mp, 0), p1 = ref_poc(e, mp, 1), q0 = ref_poc(e, mq, 0), q1 = ref_poc(e, mq, 1);
        int same = p0 == q0 && p1 == q1, swp = p0 == q1 && p1 == q0;
        if (!same && !swp) return 1;
        int o1 = !mv_far(mp->mv[0], mq->mv[0]) && !mv_far(mp->mv[1], mq->mv[1]);
        int o2 = !mv_far(mp->mv[0], mq->mv[1]) && !mv_far(mp->mv[1], mq->mv[0]);
        if (same && !swp) return !o1;
        if (!same && swp) return !o2;
        return !(o1 || o2);
    }
    return 0;
}

static int excluded(const dbk_env_t* e, int x, int y, int vert) {
    if (vert ? x == 0 : y == 0) return 1;
    int aq = (y / e->ctb) * e->wctb + x / e->ctb;
    const hevc_slice_t* sq = slice_of(e, aq);
    if (sq->deblocking_disabled) return 1;
    int ap = vert ? (y / e->ctb) * e->wctb + (x - 1) / e->ctb : ((y - 1) / e->ctb) * e->wctb + x / e->ctb;
    const hevc_pic_params_t* p = &e->syn->params;
    if (p->tiles_enabled && !p->loop_filter_across_tiles && e->syn->ctb_tile &&
        e->syn->ctb_tile[aq] != e->syn->ctb_tile[ap])
        return 1;
    int sl_q = e->syn->ctb_slice ? e->syn->ctb_slice[aq] : 0;
    int sl_p = e->syn->ctb_slice ? e->syn->ctb_slice[ap] : 0;
    if (sl_q != sl_p && !sq->lf_across_slices) return 1;
    return 0;
}

static void deblock(const hevc_picture_syntax_t* syn, planes_t* pic) {
    dbk_env_t e;
    e.syn = syn;
    e.W = syn->params.width;
    e.H = syn->params.height;
    e.gw = e.W / 4;
    e.ctb = 1 << syn->params.log2_ctb;
    e.wctb = (e.W + e.ctb - 1) / e.ctb;
    e.mot = (mot_t*)calloc((size_t)e.gw * (e.H / 4), sizeof(mot_t));
    for (size_t i = 0; i < (size_t)e.gw * (e.H / 4); i++) e.mot[i].ref[0] = e.mot[i].ref[1] = -1;
    for (int i = 0; i < syn->num_pus; i++) {
        const hevc_pu_t* pu = &syn->pus[i];
        for (int y = pu->y; y < pu->y + pu->h; y += 4)
            for (int x = pu->x; x < pu->x + pu->w; x += 4) {
                mot_t* m = &e.mot[(size_t)(y / 4) * e.gw + x / 4];
                memcpy(m->mv, pu->mv, sizeof(m->mv));
                m->ref[0] = pu->ref_idx[0];
                m->ref[1] = pu->ref_idx[1];
            }
    }
    int pcm_off = syn->params.pcm_loop_filter_disabled;
    uint8_t* L = pic->p[0];
    int Ls = pic->w[0];
    for (int pass = 0; pass < 2; pass++) {
        int vert = pass == 0;
        for (int ye = 0; ye < e.H; ye += 8)
            for (int xe = 0; xe < e.W; xe += 8)
                for (int seg = 0; seg < 2; seg++) {
                    int x = vert ? xe : xe + 4 * seg, y = vert ? ye + 4 * seg : ye;
                    if (x >= e.W || y >= e.H) continue;
                    if (!(blk_at(&e, x, y) & (vert ? HEVC_BLK_EDGE_V : HEVC_BLK_EDGE_H))) continue;
                    if (excluded(&e, x, y, vert)) continue;
                    int xp = vert ? x - 1 : x, yp = vert ? y : y - 1;
                    int bs = derive_bs(&e, xp, yp, x, y);
                    if (!bs) continue;
                    uint32_t bP = blk_at(&e, xp, yp), bQ = blk_at(&e, x, y);
                    int qpP = (int8_t)(bP >> HEVC_BLK_QP_SHIFT), qpQ = (int8_t)(bQ >> HEVC_BLK_QP_SHIFT);
                    int pcmP = !!(bP & HEVC_BLK_PCM), pcmQ = !!(bQ & HEVC_BLK_PCM);
                    int bypP = !!(bP & HEVC_BLK_BYPASS), bypQ = !!(bQ & HEVC_BLK_BYPASS);
                    int noP = (pcm_off && pcmP) || bypP, noQ = (pcm_off && pcmQ) || bypQ;
                    const hevc_slice_t* sq = slice_of(&e, (y / e.ctb) * e.wctb + x / e.ctb);
                    int qpl = (qpQ + qpP + 1) >> 1;
                    int beta = kBeta[CLIP3(0, 51, qpl + 2 * sq->beta_offset_div2)];
                    int tc = kTc[CLIP3(0, 53, qpl + 2 * (bs - 1) + 2 * sq->tc_offset_div2)];
                    /* sample (i along the filter, k along the edge): P side i = -1-i */
#define LS(i, k) (vert ? &L[(size_t)(y + (k)) * Ls + x + (i)] : &L[(size_t)(y + (i)) * Ls + x + (k)])
                    int dp0 = abs(*LS(-3, 0) - 2 * *LS(-2, 0) + *LS(-1, 0));
                    int dp3 = abs(*LS(-3, 3) - 2 * *LS(-2, 3) + *LS(-1, 3));
                    int dq0 = abs(*LS(2, 0) - 2 * *LS(1, 0) + *LS(0, 0));
                    int dq3 = abs(*LS(2, 3) - 2 * *LS(1, 3) + *LS(0, 3));
                    int dpq0 = dp0 + dq0, dpq3 = dp3 + dq3, dp = dp0 + dp3, dq = dq0 + dq3;
                    int d = dpq0 + dpq3;
                    if (d < beta) {
                        int strong = 1;
                        for (int kk = 0; kk < 2; kk++) {
                            int k = kk * 3, dpq = kk ? dpq3 : dpq0;
                            int p0 = *LS(-1, k), p3 = *LS(-4, k), q0 = *LS(0, k), q3 = *LS(3, k);
                            if (!(2 * dpq < (beta >> 2) && abs(p3 - p0) + abs(q0 - q3) < (beta >> 3) &&
                                  abs(p0 - q0) < ((5 * tc + 1) >> 1)))
                                strong = 0;
                        }
                        int side_thr = (beta + (beta >> 1)) >> 3;
                        int dEp = dp < side_thr, dEq = dq < side_thr;
                        for (int k = 0; k < 4; k++) {
                            int p[4], q[4];
                            for (int i = 0; i < 4; i++) { p[i] = *LS(-1 - i, k); q[i] = *LS(i, k); }
                            int po[3] = {p[0], p[1], p[2]}, qo[3] = {q[0], q[1], q[2]};
                            int np = 0, nq = 0;
                            if (strong) {
                                np = nq = 3;
                                int t2 = 2 * tc;
                                po[0] = CLIP3(p[0] - t2, p[0] + t2, (p[2] + 2 * p[1] + 2 * p[0] + 2 * q[0] + q[1] + 4) >> 3);
                                po[1] = CLIP3(p[1] - t2, p[1] + t2, (p[2] + p[1] + p[0] + q[0] + 2) >> 2);
                                po[2] = CLIP3(p[2] - t2, p[2] + t2, (2 * p[3] + 3 * p[2] + p[1] + p[0] + q[0] + 4) >> 3);
                                qo[0] = CLIP3(q[0] - t2, q[0] + t2, (p[1] + 2 * p[0] + 2 * q[0] + 2 * q[1] + q[2] + 4) >> 3);
                                qo[1] = CLIP3(q[1] - t2, q[1] + t2, (p[0] + q[0] + q[1] + q[2] + 2) >> 2);
                                qo[2] = CLIP3(q[2] - t2, q[2] + t2, (p[0] + q[0] + q[1] + 3 * q[2] + 2 * q[3] + 4) >> 3);
                            } else {
                                int delta = (9 * (q[0] - p[0]) - 3 * (q[1] - p[1]) + 8) >> 4;
                                if (abs(delta) < tc * 10) {
                                    delta = CLIP3(-tc, tc, delta);
                                    po[0] = CLIP3(0, 255, p[0] + delta);
                                    qo[0] = CLIP3(0, 255, q[0] - delta);
                                    if (dEp) po[1] = CLIP3(0, 255, p[1] + CLIP3(-(tc >> 1), tc >> 1, (((p[2] + p[0] + 1) >> 1) - p[1] + delta) >> 1));
                                    if (dEq) qo[1] = CLIP3(0, 255, q[1] + CLIP3(-(tc >> 1), tc >> 1, (((q[2] + q[0] + 1) >> 1) - q[1] - delta) >> 1));
                                    np = dEp + 1;
                                    nq = dEq + 1;
                                }
                            }
                            if (noP) np = 0;
                            if (noQ) nq = 0;
                            for (int i = 0; i < np; i++) *LS(-1 - i, k) = (uint8_t)po[i];
                            for (int i = 0; i < nq; i++) *LS(i, k) = (uint8_t)qo[i];
                        }
                    }
#undef LS
                    /* chroma: Bs 2 and on the 8-sample chroma grid (:538-609) */
                    if (bs == 2 && (((vert ? x : y) / 2) % 8) == 0) {
                        for (int ci = 1; ci <= 2; ci++) {
                            int off = ci == 1 ? syn->params.cb_qp_offset : syn->params.cr_qp_offset;
                            int qpi = ((qpQ + qpP + 1) >> 1) + off;
                            int qpc = kQpc[CLIP3(0, 57, qpi)];
                            int tcc = kTc[CLIP3(0, 53, qpc + 2 + 2 * sq->tc_offset_div2)];
                            uint8_t* C = pic->p[ci];
                            int Cs = pic->w[ci];
                            int cx = x / 2, cy = y / 2;
                            for (int k = 0; k < 2; k++) {
#define CS(i) (vert ? &C[(size_t)(cy + k) * Cs + cx + (i)] : &C[(size_t)(cy + (i)) * Cs + cx + k])
                                int p0 = *CS(-1), p1 = *CS(-2), q0 = *CS(0), q1 = *CS(1);
                                int delta = CLIP3(-tcc, tcc, ((((q0 - p0) * 4) + p1 - q1 + 4) >> 3));
                                if (!noP) *CS(-1) = (uint8_t)CLIP3(0, 255, p0 + delta);
                                if (!noQ) *CS(0) = (uint8_t)CLIP3(0, 255, q0 - delta);
#undef CS
                            }
                        }
                    }
                }
    }
    free(e.mot);
}

/* ------------------------------------------------------------------------------------
 * SAO: apply_sao (sao.cpp:20-243).  Reads a copy of the deblocked picture, writes the
 * picture.  Band offset applies only for band - band_position in 0..3 (no wrap at 32,
 * sao.cpp:229-230, a deviation from H.265 that parity follows).
 * ---------------------------------------------------------------------------------- */
static void sao(const hevc_picture_syntax_t* syn, const planes_t* src, planes_t* dst) {
    static const int edx[4][2] = {{-1, 1}, {0, 0}, {-1, 1}, {1, -1}};
    static const int edy[4][2] = {{0, 0}, {-1, 1}, {-1, 1}, {-1, 1}};
    const hevc_pic_params_t* p = &syn->params;
    int ctb = 1 << p->log2_ctb;
    int wc = (p->width + ctb - 1) / ctb, hc = (p->height + ctb - 1) / ctb;
    int gw = p->width / 4;
    int pcm_off = p->pcm_loop_filter_disabled;
    for (int ry = 0; ry < hc; ry++)
        for (int rx = 0; rx < wc; rx++) {
            int addr = ry * wc + rx;
            const hevc_sao_t* s = &syn->sao[addr];
            for (int ci = 0; ci < 3; ci++) {
                if (!s->type[ci]) continue;
                int sub = ci ? 2 : 1, n = ctb / sub;
                int w = src->w[ci], h = src->h[ci];
                const uint8_t* S = src->p[ci];
                uint8_t* D = dst->p[ci];
                for (int j = 0; j < n && ry * n + j < h; j++)
                    for (int i = 0; i < n && rx * n + i < w; i++) {
                        int xs = rx * n + i, ys = ry * n + j;
                        uint32_t b = syn->blk[(size_t)(ys * sub / 4) * gw + xs * sub / 4];
                        if ((pcm_off && (b & HEVC_BLK_PCM)) || (b & HEVC_BLK_BYPASS)) continue;
                        int c = S[(size_t)ys * w + xs], v;
                        if (s->type[ci] == 2) {
                            int cl = s->eo_class[ci];
                            int ax = xs + edx[cl][0], ay = ys + edy[cl][0];
                            int bx = xs + edx[cl][1], by = ys + edy[cl][1];
                            if (ax < 0 || ay < 0 || ax >= w || ay >= h || bx < 0 || by < 0 || bx >= w || by >= h) continue;
                            int skip = 0;
                            /* cross-slice / cross-tile neighbours (sao.cpp:142-185) */
                            int cur = (ys * sub / ctb) * wc + xs * sub / ctb;
                            for (int nk = 0; nk < 2 && !skip; nk++) {
                                int nx = nk ? bx : ax, ny = nk ? by : ay;
                                int na = (ny * sub / ctb) * wc + nx * sub / ctb;
                                int sc = syn->ctb_slice ? syn->ctb_slice[cur] : 0;
                                int sn = syn->ctb_slice ? syn->ctb_slice[na] : 0;
                                if (sc != sn) {
                                    int owner = sn < sc ? cur : na;
                                    int so = syn->ctb_slice ? syn->ctb_slice[owner] : 0;
                                    if (so >= syn->num_slices) so = 0;
                                    if (!syn->slices[so].lf_across_slices) skip = 1;
                                }
                                if (!skip && p->tiles_enabled && !p->loop_filter_across_tiles && syn->ctb_tile &&
                                    syn->ctb_tile[cur] != syn->ctb_tile[na])
                                    skip = 1;
                            }
                            if (skip) continue;
                            int a = S[(size_t)ay * w + ax], bb = S[(size_t)by * w + bx];
                            int e = 2 + (c < a ? -1 : c > a) + (c < bb ? -1 : c > bb);
                            v = c + s->offset[ci][e];
                        } else {
                            int k = (c >> 3) - s->band_pos[ci];
                            if (k < 0 || k >= 4) continue;
                            v = c + s->offset[ci][k];
                        }
                        D[(size_t)ys * w + xs] = (uint8_t)CLIP3(0, 255, v);
                    }
            }
        }
}

int oracle_loop_filter(const hevc_picture_syntax_t* syn, const uint8_t* in, uint8_t* out, int do_deblock,
                       int do_sao) {
    int W = syn->params.width, H = syn->params.height;
    size_t sz = (size_t)W * H * 3 / 2;
    uint8_t* work = (uint8_t*)malloc(sz);
    if (!work) return -1;
    memcpy(work, in, sz);
    planes_t wp, op;
    planes_of(work, W, H, &wp);
    if (do_deblock) deblock(syn, &wp);
    memcpy(out, work, sz);
    if (do_sao && syn->params.sao_enabled) {
        planes_of(out, W, H, &op);
        sao(syn, &wp, &op);
    }
    free(work);
    return 0;
}

/* Whole picture: MC of every PU, residual of coded inter TUs added to it, intra TUs in
 * decode order, deblocking, SAO.  The reference interleaves these per CU in decode
 * order (coding_tree.cpp:749-1056); the stage order used here reads exactly the same
 * samples, because MC reads only reference pictures and an intra TU only reads
 * neighbours that precede it in decode order. */
int oracle_reconstruct_picture(const hevc_picture_syntax_t* syn, const uint8_t* const* refs, int32_t num_refs,
                               uint8_t* out) {
    int W = syn->params.width, H = syn->params.height;
    memset(out, 0, (size_t)W * H * 3 / 2);
    if (oracle_inter_pred(&syn->params, syn->pus, syn->num_pus, syn->wp, syn->num_wp, refs, num_refs, out))
        return -1;
    planes_t pic;
    planes_of(out, W, H, &pic);
    inter_residuals(syn, &pic);
    intra_pass(syn, &pic);
    return oracle_loop_filter(syn, out, out, 1, 1);
}
