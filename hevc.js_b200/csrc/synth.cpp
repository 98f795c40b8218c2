// synth.cpp — seeded generator of reconstruction workloads (see synth.h).
#include "synth.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

namespace {

struct Rng {
    std::mt19937_64 eng;
    explicit Rng(uint64_t seed) : eng(seed) {}
    uint64_t u64() { return eng(); }
    double unit() { return (double)(eng() >> 11) * (1.0 / 9007199254740992.0); }
    bool bern(double p) { return unit() < p; }
    int range(int lo, int hi) {  // inclusive
        uint64_t span = (uint64_t)(hi - lo + 1);
        return lo + (int)(eng() % span);
    }
    int geometric_ge1(double p) {  // number of trials to first success, >= 1
        int k = 1;
        while (!bern(p) && k < 1 << 20) k++;
        return k;
    }
};

// Chroma QP mapping of the spec table used by the hevc.js TU decode
// (qpChromaTable, src/decoding/cabac_tables.h:275; applied at coding_tree.cpp:1366-1377).
int chroma_qp_prime(int qp_y, int offset) {
    static const int8_t tab[58] = {
        0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19,
        20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 29, 30, 31, 32, 33, 33, 34, 34, 35, 35,
        36, 36, 37, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51};
    int qpi = std::min(57, std::max(0, qp_y + offset));  // QpBdOffsetC = 0 at 8 bit
    return qpi < 58 ? tab[qpi] : qpi - 6;
}

// Chroma intra mode from the coded intra_chroma_pred_mode and the luma mode
// (derive_chroma_intra_mode, coding_tree.cpp:298-309).
int chroma_mode_from(int coded, int luma_mode) {
    if (coded == 4) return luma_mode;
    static const int cand[4] = {0, 26, 10, 1};
    int m = cand[coded];
    return m == luma_mode ? 34 : m;
}

void draw_levels(Rng& r, int n, int16_t* dst) {
    for (int v = 0; v < n; v++)
        for (int u = 0; u < n; u++) {
            double p = 0.6 * std::exp(-0.25 * (double)(u + v));
            int16_t val = 0;
            if (r.bern(p)) {
                int mag = r.geometric_ge1(0.5);
                if (mag > 32767) mag = 32767;
                val = (int16_t)(r.bern(0.5) ? -mag : mag);
            }
            dst[v * n + u] = val;
        }
}

void draw_scaling(Rng& r, hevc_scaling_t* s) {
    std::memset(s, 0, sizeof(*s));
    for (int sz = 0; sz < 4; sz++)
        for (int m = 0; m < 6; m++) {
            const int n = sz == 0 ? 4 : 8, kind = r.range(0, 2), k = r.range(0, 12);
            for (int v = 0; v < n; v++)
                for (int u = 0; u < n; u++)
                    s->list[sz][m][v * n + u] =
                        (uint8_t)(kind == 0 ? 16 : kind == 1 ? 16 + k * (u + v) : r.range(0, 255));
        }
    for (int i = 0; i < 2; i++)
        for (int m = 0; m < 6; m++) s->dc[i][m] = (uint8_t)(r.bern(0.25) ? 0 : r.range(0, 255));
}

struct Picture {
    hevcsynth_picture_t pub{};
    hevc_scaling_t scaling{};
    std::vector<hevc_tu_t> tus;
    std::vector<int16_t> coeffs;
    std::vector<hevc_pu_t> pus;
    std::vector<hevc_wp_t> wp;
    std::vector<uint32_t> blk;
    std::vector<hevc_sao_t> sao;
    std::vector<uint8_t> ctb_slice;
    std::vector<uint16_t> ctb_tile;
    std::vector<hevc_slice_t> slices;
    std::vector<hevcsynth_cu_t> cus;
};

struct Gen {
    const hevcsynth_cfg_t& c;
    Rng r;
    Picture& P;
    int W, H, gw;  // gw = W/4
    hevc_pu_t last_pu{};
    bool have_last = false;
    int cu_luma_mode[4] = {1, 1, 1, 1};

    Gen(const hevcsynth_cfg_t& cfg, Picture& pic)
        : c(cfg), r(cfg.seed), P(pic), W(cfg.width), H(cfg.height), gw(cfg.width / 4) {}

    uint32_t& blk(int x, int y) { return P.blk[(size_t)(y / 4) * gw + (x / 4)]; }

    void set_tu_log2(int x0, int y0, int size, int log2, bool cbf) {
        for (int dy = 0; dy < size; dy += 4)
            for (int dx = 0; dx < size; dx += 4) {
                if (x0 + dx >= W || y0 + dy >= H) continue;
                uint32_t& b = blk(x0 + dx, y0 + dy);
                b = (b & ~(0xFFu << HEVC_BLK_TU_SHIFT) & ~HEVC_BLK_CBF) |
                    ((uint32_t)log2 << HEVC_BLK_TU_SHIFT) | (cbf ? HEVC_BLK_CBF : 0u);
            }
    }
    void edge_v(int x, int y0, int len) {
        if (x >= W) return;
        for (int dy = 0; dy < len; dy += 4)
            if (y0 + dy < H) blk(x, y0 + dy) |= HEVC_BLK_EDGE_V;
    }
    void edge_h(int x0, int y, int len) {
        if (y >= H) return;
        for (int dx = 0; dx < len; dx += 4)
            if (x0 + dx < W) blk(x0 + dx, y) |= HEVC_BLK_EDGE_H;
    }

    void emit_tu(int x, int y, int log2, int cidx, int qp_prime, bool intra, int mode,
                 bool coded) {
        hevc_tu_t t{};
        t.x = (uint16_t)x;
        t.y = (uint16_t)y;
        t.log2_size = (uint8_t)log2;
        t.c_idx = (uint8_t)cidx;
        t.qp = (uint8_t)qp_prime;
        t.flags = (uint8_t)((intra ? HEVC_TU_INTRA : 0) | (coded ? HEVC_TU_CODED : 0));
        t.intra_mode = (uint8_t)mode;
        t.coeff_offset = 0;
        if (coded) {
            int n = 1 << log2;
            t.coeff_offset = (uint32_t)P.coeffs.size();
            P.coeffs.resize(P.coeffs.size() + (size_t)n * n);
            draw_levels(r, n, &P.coeffs[t.coeff_offset]);
        }
        P.tus.push_back(t);
    }

    // A PCM block: its samples (uniform 0..255) as the levels of an intra TU.
    void emit_pcm(int x, int y, int log2, int cidx, int qp) {
        hevc_tu_t t{};
        t.x = (uint16_t)x;
        t.y = (uint16_t)y;
        t.log2_size = (uint8_t)log2;
        t.c_idx = (uint8_t)cidx;
        t.qp = (uint8_t)std::max(0, qp);
        t.flags = (uint8_t)(HEVC_TU_INTRA | HEVC_TU_CODED | HEVC_TU_PCM);
        t.intra_mode = 1;
        const int n = 1 << log2;
        t.coeff_offset = (uint32_t)P.coeffs.size();
        P.coeffs.resize(P.coeffs.size() + (size_t)n * n);
        for (int i = 0; i < n * n; i++) P.coeffs[t.coeff_offset + (size_t)i] = (int16_t)r.range(0, 255);
        P.tus.push_back(t);
    }

    // Transform tree in parse order (decode_transform_tree, coding_tree.cpp:1146-1250).
    void tree(const hevcsynth_cu_t& cu, int chroma_mode, int x0, int y0, int xb, int yb,
              int log2, int depth, int blk_idx, bool cbf_cb_par, bool cbf_cr_par) {
        bool intra = cu.pred_mode == 1;
        bool nxn = intra && cu.part_mode == 3;
        bool split;
        if (log2 > 5) split = true;
        else if (nxn && depth == 0) split = true;
        else if (log2 > 2) split = r.bern(c.p_tu_split);
        else split = false;
        bool cbf_cb = cbf_cb_par, cbf_cr = cbf_cr_par;
        if (log2 > 2) {
            cbf_cb = (depth == 0 || cbf_cb_par) ? r.bern(c.p_cbf_chroma) : false;
            cbf_cr = (depth == 0 || cbf_cr_par) ? r.bern(c.p_cbf_chroma) : false;
        }
        if (split) {
            int h = 1 << (log2 - 1);
            tree(cu, chroma_mode, x0, y0, x0, y0, log2 - 1, depth + 1, 0, cbf_cb, cbf_cr);
            tree(cu, chroma_mode, x0 + h, y0, x0, y0, log2 - 1, depth + 1, 1, cbf_cb, cbf_cr);
            tree(cu, chroma_mode, x0, y0 + h, x0, y0, log2 - 1, depth + 1, 2, cbf_cb, cbf_cr);
            tree(cu, chroma_mode, x0 + h, y0 + h, x0, y0, log2 - 1, depth + 1, 3, cbf_cb, cbf_cr);
            return;
        }
        bool cbf_luma = r.bern(c.p_cbf_luma);
        int qp_y = cu.qp_y;
        int luma_mode = 1;
        if (intra) {
            int half = 1 << (cu.log2_size - 1);
            int pu = nxn ? ((y0 - cu.y) >= half ? 2 : 0) + ((x0 - cu.x) >= half ? 1 : 0) : 0;
            luma_mode = cu_luma_mode[pu];
        }
        if (intra || cbf_luma) emit_tu(x0, y0, log2, 0, qp_y, intra, luma_mode, cbf_luma);
        int log2c = std::max(2, log2 - 1);
        bool do_chroma = (log2 > 2) || (blk_idx == 3);
        int xc = (log2 == 2) ? xb : x0, yc = (log2 == 2) ? yb : y0;
        if (do_chroma) {
            for (int ci = 1; ci <= 2; ci++) {
                bool cbf = ci == 1 ? cbf_cb : cbf_cr;
                int qpc = chroma_qp_prime(qp_y, ci == 1 ? c.cb_qp_offset : c.cr_qp_offset);
                if (intra || cbf) emit_tu(xc / 2, yc / 2, log2c, ci, qpc, intra, chroma_mode, cbf);
            }
        }
        // deblocking side info of the TU leaf (coding_tree.cpp:1229-1248)
        int n = 1 << log2;
        set_tu_log2(x0, y0, n, log2, cbf_luma);
        edge_v(x0, y0, n);
        edge_h(x0, y0, n);
    }

    void emit_pu(int x, int y, int w, int h) {
        hevc_pu_t pu{};
        pu.x = (uint16_t)x;
        pu.y = (uint16_t)y;
        pu.w = (uint8_t)w;
        pu.h = (uint8_t)h;
        pu.wp = -1;
        if (have_last && r.bern(c.p_merge)) {
            pu.ref_idx[0] = last_pu.ref_idx[0];
            pu.ref_idx[1] = last_pu.ref_idx[1];
            std::memcpy(pu.mv, last_pu.mv, sizeof(pu.mv));
            pu.wp = last_pu.wp;
            if (w + h == 12 && pu.ref_idx[0] >= 0 && pu.ref_idx[1] >= 0) pu.ref_idx[1] = -1;
        } else {
            bool small = (w + h == 12);  // 8x4 / 4x8 stay uni-predicted
            bool bi = c.slice_type == 0 && !small && r.bern(c.p_bi);
            int list = (c.slice_type == 0 && r.bern(0.5)) ? 1 : 0;
            for (int l = 0; l < 2; l++) {
                bool use = bi || l == list;
                pu.ref_idx[l] = (int8_t)(use ? r.range(0, c.num_refs - 1) : -1);
                pu.mv[l][0] = (int16_t)(use ? r.range(-c.mv_range, c.mv_range) : 0);
                pu.mv[l][1] = (int16_t)(use ? r.range(-c.mv_range, c.mv_range) : 0);
            }
            if (r.bern(c.p_wp)) {
                hevc_wp_t w8{};
                w8.log2wd[0] = 6 + 6;  // luma_log2_weight_denom 6 + shift1 6
                w8.log2wd[1] = 6 + 6;
                for (int l = 0; l < 2; l++)
                    for (int ci = 0; ci < 3; ci++) {
                        w8.w[l][ci] = (int16_t)r.range(32, 96);
                        w8.o[l][ci] = (int16_t)r.range(-16, 16);
                    }
                pu.wp = (int16_t)P.wp.size();
                P.wp.push_back(w8);
            }
        }
        P.pus.push_back(pu);
        last_pu = pu;
        have_last = true;
    }

    void coding_unit(int x0, int y0, int log2) {
        hevcsynth_cu_t cu{};
        cu.x = (uint16_t)x0;
        cu.y = (uint16_t)y0;
        cu.log2_size = (uint8_t)log2;
        int n = 1 << log2;
        bool intra = c.slice_type == 2 || r.bern(c.p_intra);
        cu.pred_mode = intra ? 1 : 0;
        cu.qp_y = (int8_t)r.range(c.qp_min, c.qp_max);
        if (!intra && r.bern(c.p_skip)) cu.pred_mode = 2;
        int part = 0;
        if (intra) {
            part = (log2 == 3 && r.bern(c.p_intra_nxn)) ? 3 : 0;
        } else if (cu.pred_mode == 0) {
            int k = r.range(0, 3);  // 2Nx2N, 2NxN, Nx2N, AMP
            if (k == 3) part = log2 == 3 ? 0 : 4 + r.range(0, 3);
            else part = k;
        }
        cu.part_mode = (uint8_t)part;
        cu.first_pu = (int32_t)P.pus.size();
        if (!intra) {
            int h2 = n / 2, q = n / 4;
            switch (part) {
                case 0: emit_pu(x0, y0, n, n); break;
                case 1: emit_pu(x0, y0, n, h2); emit_pu(x0, y0 + h2, n, h2); break;
                case 2: emit_pu(x0, y0, h2, n); emit_pu(x0 + h2, y0, h2, n); break;
                case 4: emit_pu(x0, y0, n, q); emit_pu(x0, y0 + q, n, n - q); break;
                case 5: emit_pu(x0, y0, n, n - q); emit_pu(x0, y0 + n - q, n, q); break;
                case 6: emit_pu(x0, y0, q, n); emit_pu(x0 + q, y0, n - q, n); break;
                case 7: emit_pu(x0, y0, n - q, n); emit_pu(x0 + n - q, y0, q, n); break;
            }
        }
        cu.num_pu = (int32_t)P.pus.size() - cu.first_pu;
        // PCM (pcm_flag of a 2Nx2N intra CU, coding_tree.cpp:1425-1469); drawn only when asked,
        // so that the pictures of other settings stay the same
        const bool pcm = intra && part == 0 && log2 <= 5 && c.p_pcm > 0 && r.bern(c.p_pcm);

        // CU-level grid initialisation (coding_tree.cpp:960-1021)
        uint32_t base = (intra ? HEVC_BLK_INTRA : 0u) | (pcm ? HEVC_BLK_PCM : 0u) |
                        ((uint32_t)(uint8_t)cu.qp_y << HEVC_BLK_QP_SHIFT) |
                        ((uint32_t)log2 << HEVC_BLK_TU_SHIFT);
        for (int dy = 0; dy < n; dy += 4)
            for (int dx = 0; dx < n; dx += 4) {
                uint32_t& b = blk(x0 + dx, y0 + dy);
                b = (b & (HEVC_BLK_EDGE_V | HEVC_BLK_EDGE_H)) | base;
            }
        edge_v(x0, y0, n);
        edge_h(x0, y0, n);
        if (part == 2 || part == 3) edge_v(x0 + n / 2, y0, n);
        if (part == 6) edge_v(x0 + n / 4, y0, n);
        if (part == 7) edge_v(x0 + 3 * n / 4, y0, n);
        if (part == 1 || part == 3) edge_h(x0, y0 + n / 2, n);
        if (part == 4) edge_h(x0, y0 + n / 4, n);
        if (part == 5) edge_h(x0, y0 + 3 * n / 4, n);

        int chroma_mode = 0;
        if (intra) {
            int npu = part == 3 ? 4 : 1;
            for (int i = 0; i < npu; i++) cu_luma_mode[i] = r.range(0, 34);
            chroma_mode = chroma_mode_from(r.range(0, 4), cu_luma_mode[0]);
        }
        cu.first_tu = (int32_t)P.tus.size();
        cu.has_tree = cu.pred_mode != 2 && !pcm;
        if (pcm) {   // the samples in decode order: luma, then Cb and Cr
            emit_pcm(x0, y0, log2, 0, cu.qp_y);
            emit_pcm(x0 / 2, y0 / 2, log2 - 1, 1, cu.qp_y);
            emit_pcm(x0 / 2, y0 / 2, log2 - 1, 2, cu.qp_y);
        }
        if (cu.has_tree) tree(cu, chroma_mode, x0, y0, x0, y0, log2, 0, 0, true, true);
        cu.num_tu = (int32_t)P.tus.size() - cu.first_tu;
        P.cus.push_back(cu);
    }

    void quadtree(int x0, int y0, int log2) {
        if (x0 >= W || y0 >= H) return;
        int n = 1 << log2;
        bool inside = x0 + n <= W && y0 + n <= H;
        bool split;
        if (log2 <= 3) split = false;
        else if (!inside) split = true;
        else split = r.bern(c.p_split);
        if (split) {
            int h = n / 2;
            quadtree(x0, y0, log2 - 1);
            quadtree(x0 + h, y0, log2 - 1);
            quadtree(x0, y0 + h, log2 - 1);
            quadtree(x0 + h, y0 + h, log2 - 1);
        } else {
            coding_unit(x0, y0, log2);
        }
    }

    void sao_params(hevc_sao_t& s) {
        std::memset(&s, 0, sizeof(s));
        int chroma_type = 0, chroma_class = 0;
        for (int ci = 0; ci < 3; ci++) {
            int type;
            if (ci == 2) type = chroma_type;
            else {
                double u = r.unit();
                type = u < 0.3 ? 0 : (u < 0.6 ? 1 : 2);
            }
            if (ci == 1) chroma_type = type;
            s.type[ci] = (uint8_t)type;
            if (type == 0) continue;
            int a[4];
            for (int i = 0; i < 4; i++) a[i] = r.range(0, 7);
            if (type == 1) {
                for (int i = 0; i < 4; i++) s.offset[ci][i] = (int8_t)(r.bern(0.5) ? -a[i] : a[i]);
                s.offset[ci][4] = 0;
                s.band_pos[ci] = (uint8_t)r.range(0, 31);
            } else {
                if (ci == 0) s.eo_class[0] = (uint8_t)r.range(0, 3);
                if (ci == 1) chroma_class = r.range(0, 3);
                if (ci >= 1) s.eo_class[ci] = (uint8_t)chroma_class;
                s.offset[ci][0] = (int8_t)a[0];
                s.offset[ci][1] = (int8_t)a[1];
                s.offset[ci][2] = 0;
                s.offset[ci][3] = (int8_t)-a[2];
                s.offset[ci][4] = (int8_t)-a[3];
            }
        }
    }

    void run() {
        const int log2_ctb = c.log2_ctb ? c.log2_ctb : 6;
        int ctb = 1 << log2_ctb;
        int wc = (W + ctb - 1) / ctb, hc = (H + ctb - 1) / ctb;
        P.blk.assign((size_t)(W / 4) * (H / 4), (uint32_t)log2_ctb << HEVC_BLK_TU_SHIFT);
        P.sao.assign((size_t)wc * hc, hevc_sao_t{});
        P.ctb_slice.assign((size_t)wc * hc, 0);
        // tiles with uniform spacing (column i spans CTB columns i*wc/tc .. (i+1)*wc/tc - 1);
        // the CTBs of a tile are decoded in raster order, the tiles in raster order
        const int tc = std::max(1, std::min(c.tile_cols, wc)), tr = std::max(1, std::min(c.tile_rows, hc));
        const bool tiles = tc * tr > 1;
        P.ctb_tile.assign((size_t)wc * hc, 0);
        for (int ty = 0; ty < tr; ty++)
            for (int tx = 0; tx < tc; tx++)
                for (int ry = ty * hc / tr; ry < (ty + 1) * hc / tr; ry++)
                    for (int rx = tx * wc / tc; rx < (tx + 1) * wc / tc; rx++) {
                        P.ctb_tile[(size_t)ry * wc + rx] = (uint16_t)(ty * tc + tx);
                        if (c.sao) sao_params(P.sao[(size_t)ry * wc + rx]);
                        quadtree(rx * ctb, ry * ctb, log2_ctb);
                    }
        hevc_slice_t s{};
        s.beta_offset_div2 = (int8_t)c.beta_offset_div2;
        s.tc_offset_div2 = (int8_t)c.tc_offset_div2;
        s.deblocking_disabled = 0;
        s.lf_across_slices = 1;
        P.slices.assign(1, s);

        hevc_picture_syntax_t& syn = P.pub.syn;
        std::memset(&syn, 0, sizeof(syn));
        hevc_pic_params_t& p = syn.params;
        p.width = W;
        p.height = H;
        p.bit_depth = 8;
        p.log2_ctb = log2_ctb;
        p.log2_min_cb = 3;
        p.log2_min_tb = 2;
        p.strong_intra_smoothing = c.strong_intra_smoothing;
        p.intra_smoothing_disabled = 0;
        p.pcm_loop_filter_disabled = 0;
        p.sao_enabled = c.sao ? 1 : 0;
        p.cb_qp_offset = c.cb_qp_offset;
        p.cr_qp_offset = c.cr_qp_offset;
        p.tiles_enabled = tiles ? 1 : 0;
        p.loop_filter_across_tiles = c.no_lf_across_tiles ? 0 : 1;
        int nref = c.slice_type == 2 ? 0 : c.num_refs;
        for (int l = 0; l < 2; l++) {
            p.num_ref[l] = (l == 1 && c.slice_type != 0) ? 0 : nref;
            for (int i = 0; i < 16; i++) {
                p.ref_poc[l][i] = -999999;
                p.ref_slot[l][i] = -1;
            }
            // L0 = {0, 1, ...}, L1 = {1, 0, ...}: reference slot i has POC poc-1-i.
            for (int i = 0; i < p.num_ref[l]; i++) {
                int slot = (l == 0) ? i : (nref - 1 - i);
                p.ref_slot[l][i] = slot;
                p.ref_poc[l][i] = c.poc - 1 - slot;
            }
        }
        syn.num_tus = (int32_t)P.tus.size();
        syn.tus = P.tus.data();
        syn.num_coeffs = P.coeffs.size();
        syn.coeffs = P.coeffs.data();
        syn.num_pus = (int32_t)P.pus.size();
        syn.pus = P.pus.data();
        syn.num_wp = (int32_t)P.wp.size();
        syn.wp = P.wp.data();
        syn.blk = P.blk.data();
        syn.sao = P.sao.data();
        syn.ctb_slice = P.ctb_slice.data();
        syn.ctb_tile = tiles ? P.ctb_tile.data() : nullptr;
        syn.num_slices = 1;
        syn.slices = P.slices.data();
        syn.scaling = nullptr;
        if (c.scaling_lists) {   // own stream of draws: the rest of the picture is unchanged
            Rng rs(c.seed ^ 0x5CA1E11575ull);
            draw_scaling(rs, &P.scaling);
            syn.scaling = &P.scaling;
        }
        P.pub.num_cus = (int32_t)P.cus.size();
        P.pub.cus = P.cus.data();
        P.pub.impl = &P;
    }
};

}  // namespace

extern "C" {

void hevcsynth_default_cfg(hevcsynth_cfg_t* c, int32_t width, int32_t height, uint64_t seed) {
    std::memset(c, 0, sizeof(*c));
    c->width = width;
    c->height = height;
    c->seed = seed;
    c->p_split = 0.5;
    c->p_intra = 0.0;
    c->p_intra_nxn = 0.25;
    c->p_skip = 0.0;
    c->p_bi = 0.5;
    c->p_wp = 0.1;
    c->p_merge = 0.0;
    c->mv_range = 256;
    c->p_tu_split = 0.5;
    c->p_cbf_luma = 0.6;
    c->p_cbf_chroma = 0.4;
    c->qp_min = 22;
    c->qp_max = 37;
    c->sao = 1;
    c->num_refs = 2;
    c->slice_type = 0;
    c->poc = 8;
    c->strong_intra_smoothing = 1;
    c->cb_qp_offset = 0;
    c->cr_qp_offset = 0;
}

hevcsynth_picture_t* hevcsynth_picture(const hevcsynth_cfg_t* cfg) {
    if (!cfg || cfg->width <= 0 || cfg->height <= 0 || (cfg->width & 7) || (cfg->height & 7) ||
        cfg->width > 8192 || cfg->height > 4352 || cfg->num_refs < 1 || cfg->num_refs > 2 ||
        cfg->qp_min < 0 || cfg->qp_max > 51 || cfg->qp_min > cfg->qp_max ||
        (cfg->log2_ctb != 0 && (cfg->log2_ctb < 4 || cfg->log2_ctb > 6)))
        return nullptr;
    Picture* P = new Picture();
    Gen g(*cfg, *P);
    g.run();
    return &P->pub;
}

void hevcsynth_picture_free(hevcsynth_picture_t* pic) {
    if (!pic) return;
    delete static_cast<Picture*>(pic->impl);
}

int hevcsynth_content(int32_t width, int32_t height, uint64_t seed, uint8_t* out) {
    if (!out || width <= 0 || height <= 0 || (width & 1) || (height & 1)) return -1;
    Rng r(seed);
    const double two_pi = 6.283185307179586;
    uint8_t* plane = out;
    for (int ci = 0; ci < 3; ci++) {
        int w = ci ? width / 2 : width, h = ci ? height / 2 : height;
        double fx[8], fy[8], ph[8], amp[8];
        for (int k = 0; k < 8; k++) {
            double period = 8.0 + r.unit() * 248.0;
            double theta = r.unit() * two_pi;
            fx[k] = std::cos(theta) * two_pi / period;
            fy[k] = std::sin(theta) * two_pi / period;
            ph[k] = r.unit() * two_pi;
            amp[k] = 6.0 + r.unit() * 18.0;
        }
        // sin(a + b) = sin a cos b + cos a sin b with a = fx*x (per column) and
        // b = fy*y + phase (per row): two tables per sinusoid instead of a sin per sample
        std::vector<double> sx((size_t)8 * w), cx((size_t)8 * w), sy((size_t)8 * h), cy((size_t)8 * h);
        for (int k = 0; k < 8; k++) {
            for (int x = 0; x < w; x++) {
                sx[(size_t)k * w + x] = amp[k] * std::sin(fx[k] * x);
                cx[(size_t)k * w + x] = amp[k] * std::cos(fx[k] * x);
            }
            for (int y = 0; y < h; y++) {
                sy[(size_t)k * h + y] = std::sin(fy[k] * y + ph[k]);
                cy[(size_t)k * h + y] = std::cos(fy[k] * y + ph[k]);
            }
        }
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                double v = 128.0;
                for (int k = 0; k < 8; k++)
                    v += sx[(size_t)k * w + x] * cy[(size_t)k * h + y] + cx[(size_t)k * w + x] * sy[(size_t)k * h + y];
                int s = (int)std::lround(v) + r.range(-8, 8);
                plane[(size_t)y * w + x] = (uint8_t)std::min(255, std::max(0, s));
            }
        plane += (size_t)w * h;
    }
    return 0;
}

int hevcsynth_scaling(uint64_t seed, hevc_scaling_t* out) {
    if (!out) return -1;
    Rng r(seed);
    draw_scaling(r, out);
    return 0;
}

int64_t hevcsynth_blocks(int32_t num_tus, uint64_t seed, int32_t qp_min, int32_t qp_max,
                         hevc_tu_t* tus, int16_t* coeffs, uint8_t* pred) {
    if (num_tus < 0 || qp_min < 0 || qp_max > 51 || qp_min > qp_max) return -1;
    Rng r(seed);
    int64_t off = 0;
    for (int t = 0; t < num_tus; t++) {
        double u = r.unit();
        int log2 = 2;
        bool dst = false;
        if (u < 0.25) { log2 = 2; dst = true; }
        else if (u < 0.50) log2 = 2;
        else if (u < 0.75) log2 = 3;
        else if (u < 0.90) log2 = 4;
        else log2 = 5;
        int qp = r.range(qp_min, qp_max);
        int n = 1 << log2;
        if (tus) {
            hevc_tu_t& t0 = tus[t];
            std::memset(&t0, 0, sizeof(t0));
            t0.log2_size = (uint8_t)log2;
            t0.c_idx = 0;
            t0.qp = (uint8_t)qp;
            t0.flags = (uint8_t)(HEVC_TU_CODED | (dst ? HEVC_TU_INTRA : 0));
            t0.coeff_offset = (uint32_t)off;
        }
        if (coeffs) {
            draw_levels(r, n, coeffs + off);
        } else {
            std::vector<int16_t> scratch((size_t)n * n);
            draw_levels(r, n, scratch.data());
        }
        for (int i = 0; i < n * n; i++) {
            int v = r.range(0, 255);
            if (pred) pred[off + i] = (uint8_t)v;
        }
        off += (int64_t)n * n;
    }
    return off;
}

int hevcsynth_bs_histogram(const hevc_picture_syntax_t* syn, int64_t counts[3]) {
    if (!syn || !counts) return -1;
    counts[0] = counts[1] = counts[2] = 0;
    const hevc_pic_params_t& p = syn->params;
    int W = p.width, H = p.height, gw = W / 4, gh = H / 4;
    // motion grid from the PUs
    struct M { int16_t mv[2][2]; int8_t ref[2]; };
    std::vector<M> mot((size_t)gw * gh, M{{{0, 0}, {0, 0}}, {-1, -1}});
    for (int i = 0; i < syn->num_pus; i++) {
        const hevc_pu_t& pu = syn->pus[i];
        for (int y = pu.y; y < pu.y + pu.h; y += 4)
            for (int x = pu.x; x < pu.x + pu.w; x += 4) {
                M& m = mot[(size_t)(y / 4) * gw + x / 4];
                std::memcpy(m.mv, pu.mv, sizeof(m.mv));
                m.ref[0] = pu.ref_idx[0];
                m.ref[1] = pu.ref_idx[1];
            }
    }
    auto poc = [&](const M& m, int l) -> int {
        int ri = m.ref[l];
        if (ri < 0 || ri >= p.num_ref[l]) return -999999;
        return p.ref_poc[l][ri];
    };
    auto bs_of = [&](int xp, int yp, int xq, int yq) -> int {
        uint32_t bp = syn->blk[(size_t)(yp / 4) * gw + xp / 4];
        uint32_t bq = syn->blk[(size_t)(yq / 4) * gw + xq / 4];
        if ((bp | bq) & HEVC_BLK_INTRA) return 2;
        int tp = 1 << ((bp >> HEVC_BLK_TU_SHIFT) & 0xFF), tq = 1 << ((bq >> HEVC_BLK_TU_SHIFT) & 0xFF);
        bool tu_edge = (xp != xq) ? ((xq % tq == 0) || ((xp + 1) % tp == 0 && xp + 1 == xq))
                                  : ((yq % tq == 0) || ((yp + 1) % tp == 0 && yp + 1 == yq));
        if (tu_edge && ((bp | bq) & HEVC_BLK_CBF)) return 1;
        const M& mp = mot[(size_t)(yp / 4) * gw + xp / 4];
        const M& mq = mot[(size_t)(yq / 4) * gw + xq / 4];
        int np = (mp.ref[0] >= 0) + (mp.ref[1] >= 0), nq = (mq.ref[0] >= 0) + (mq.ref[1] >= 0);
        if (np != nq) return 1;
        auto far = [](const int16_t* a, const int16_t* b) {
            return std::abs(a[0] - b[0]) >= 4 || std::abs(a[1] - b[1]) >= 4;
        };
        if (np == 1) {
            int lp = mp.ref[0] >= 0 ? 0 : 1, lq = mq.ref[0] >= 0 ? 0 : 1;
            if (poc(mp, lp) != poc(mq, lq)) return 1;
            return far(mp.mv[lp], mq.mv[lq]) ? 1 : 0;
        }
        if (np == 2) {
            int p0 = poc(mp, 0), p1 = poc(mp, 1), q0 = poc(mq, 0), q1 = poc(mq, 1);
            bool same = p0 == q0 && p1 == q1, swp = p0 == q1 && p1 == q0;
            if (!same && !swp) return 1;
            bool o1 = !far(mp.mv[0], mq.mv[0]) && !far(mp.mv[1], mq.mv[1]);
            bool o2 = !far(mp.mv[0], mq.mv[1]) && !far(mp.mv[1], mq.mv[0]);
            if (same && !swp) return o1 ? 0 : 1;
            if (!same && swp) return o2 ? 0 : 1;
            return (o1 || o2) ? 0 : 1;
        }
        return 0;
    };
    for (int pass = 0; pass < 2; pass++)
        for (int y = 0; y < H; y += 4)
            for (int x = 0; x < W; x += 4) {
                if (pass == 0 ? (x % 8) : (y % 8)) continue;
                if (pass == 0 ? x == 0 : y == 0) continue;
                uint32_t b = syn->blk[(size_t)(y / 4) * gw + x / 4];
                if (!(b & (pass == 0 ? HEVC_BLK_EDGE_V : HEVC_BLK_EDGE_H))) continue;
                int bs = pass == 0 ? bs_of(x - 1, y, x, y) : bs_of(x, y - 1, x, y);
                counts[bs]++;
            }
    return 0;
}

}  // extern "C"
