// ref_harness.cpp — drives privaloops/hevc.js's own reconstruction functions on the
// records of include/hevcgpu.h.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with the reference's
// sources (compiled where they lie, never copied) into oracle/_ref/libhevcref.so.  It is
// used to pin the CPU restatement (oracle/hevc_oracle.c), to generate the golden digests
// under tests/golden/, and as the "reference" CPU baseline of bench.py.
//
// Every sample operation below is a call into the reference: perform_dequant and
// perform_transform_inverse (src/decoding/transform.cpp:293, :374),
// perform_intra_prediction (src/decoding/intra_prediction.cpp:428),
// perform_inter_prediction (src/decoding/interpolation.cpp:306), apply_deblocking
// (src/filters/deblocking.cpp:357) and apply_sao (src/filters/sao.cpp:20).  The harness
// only fills a DecodingContext the way src/decoding/decoder.cpp:117-185 does and stores
// results the way src/decoding/coding_tree.cpp does (add-and-clip of reconstruct_block
// :371-396; PU sample store :892-922).
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "common/picture.h"
#include "common/types.h"
#include "decoding/coding_tree.h"
#include "decoding/interpolation.h"
#include "decoding/intra_prediction.h"
#include "decoding/transform.h"
#include "filters/deblocking.h"
#include "filters/sao.h"
#include "syntax/pps.h"
#include "syntax/slice_header.h"
#include "syntax/sps.h"
// RefPicList storage of the DPB is private; the harness sets it directly.
#define private public
#include "decoding/dpb.h"
#undef private

#include "../include/hevcgpu.h"
#include "../hevc.js_b200/csrc/synth.h"

using namespace hevc;

namespace {

struct Env {
    SPS sps;
    PPS pps;
    SliceHeader sh;
    std::vector<SliceHeader> slices;
    std::vector<const SliceHeader*> slice_ptrs;
    DPB dpb;
    std::vector<std::unique_ptr<Picture>> refs;
    Picture pic;
    std::vector<CUInfo> cu_info;
    std::vector<PUMotionInfo> motion;
    std::vector<uint8_t> cbf, tu_log2, edge_v, edge_h, slice_idx;
    std::vector<DecodingContext::SaoParams> sao;
    std::vector<uint16_t> sao_backup[3];
    // the PPS and slice header a PU's weighted prediction selects, built once per (WP row,
    // refIdxL0, refIdxL1) of the picture (the default form under the key (-1, 0, 0))
    std::map<std::tuple<int, int, int>, std::pair<PPS, SliceHeader>> wp_forms;
    DecodingContext ctx;
    int W = 0, H = 0;
};

void init_sps(SPS& s, int W, int H, int log2_ctb, int log2_min_cb, int strong, int smooth_off, int pcm_lf_off,
              int sao_on) {
    s.chroma_format_idc = 1;
    s.pic_width_in_luma_samples = (uint32_t)W;
    s.pic_height_in_luma_samples = (uint32_t)H;
    s.bit_depth_luma_minus8 = 0;
    s.bit_depth_chroma_minus8 = 0;
    s.log2_min_luma_coding_block_size_minus3 = (uint32_t)(log2_min_cb - 3);
    s.log2_diff_max_min_luma_coding_block_size = (uint32_t)(log2_ctb - log2_min_cb);
    s.log2_min_luma_transform_block_size_minus2 = 0;
    s.log2_diff_max_min_luma_transform_block_size = 3;
    s.strong_intra_smoothing_enabled_flag = strong != 0;
    s.intra_smoothing_disabled_flag = smooth_off != 0;
    s.pcm_loop_filter_disabled_flag = pcm_lf_off != 0;
    s.sample_adaptive_offset_enabled_flag = sao_on != 0;
    s.scaling_list_enabled_flag = false;
    s.derive();
}

// Scaling lists: the SPS carries them (scaling_list_enabled_flag with the SPS's own
// ScalingListData; the PPS has none), as the parser leaves them (sps.cpp:400-410).
void set_scaling(SPS& s, const hevc_scaling_t* sl) {
    s.scaling_list_enabled_flag = sl != nullptr;
    if (!sl) return;
    for (int sz = 0; sz < 4; sz++)
        for (int m = 0; m < 6; m++)
            std::memcpy(s.scaling_list_data.scaling_list[(size_t)sz][(size_t)m].data(), sl->list[sz][m], 64);
    for (int i = 0; i < 2; i++)
        for (int m = 0; m < 6; m++) s.scaling_list_data.scaling_list_dc[(size_t)i][(size_t)m] = sl->dc[i][m];
}

void load_picture(Picture& pic, int W, int H, const uint8_t* i420) {
    pic.allocate(W, H, ChromaFormat::YUV420, 8, 8);
    if (!i420) return;
    const uint8_t* src = i420;
    for (int c = 0; c < 3; c++) {
        size_t n = (size_t)pic.width[c] * pic.height[c];
        for (size_t i = 0; i < n; i++) pic.planes[c][i] = src[i];
        src += n;
    }
}

void store_picture(const Picture& pic, uint8_t* i420) {
    uint8_t* dst = i420;
    for (int c = 0; c < 3; c++) {
        size_t n = (size_t)pic.width[c] * pic.height[c];
        for (size_t i = 0; i < n; i++) dst[i] = (uint8_t)pic.planes[c][i];
        dst += n;
    }
}

// Fill ctx the way decoder.cpp:117-185 does, from the records.
void setup(Env& e, const hevc_picture_syntax_t& syn, const uint8_t* in, const uint8_t* const* ref_planes,
           int num_refs) {
    const hevc_pic_params_t& p = syn.params;
    e.W = p.width;
    e.H = p.height;
    init_sps(e.sps, p.width, p.height, p.log2_ctb, p.log2_min_cb, p.strong_intra_smoothing,
             p.intra_smoothing_disabled, p.pcm_loop_filter_disabled, p.sao_enabled);
    set_scaling(e.sps, syn.scaling);
    e.pps.pps_cb_qp_offset = p.cb_qp_offset;
    e.pps.pps_cr_qp_offset = p.cr_qp_offset;
    e.pps.loop_filter_across_tiles_enabled_flag = p.loop_filter_across_tiles != 0;
    // tiles: TileId by tile-scan address with the identity scan conversion, so that
    // TileId[CtbAddrRsToTs[a]] (deblocking.cpp:79-81, sao.cpp:173-181,
    // intra_prediction.cpp:118-120) is the record's tile of raster CTB a
    e.pps.tiles_enabled_flag = p.tiles_enabled != 0 && syn.ctb_tile;
    e.pps.CtbAddrRsToTs.clear();
    e.pps.TileId.clear();
    if (e.pps.tiles_enabled_flag) {
        const int n = e.sps.PicSizeInCtbsY;
        for (int a = 0; a < n; a++) {
            e.pps.CtbAddrRsToTs.push_back(a);
            e.pps.TileId.push_back(syn.ctb_tile[a]);
        }
    }
    e.pps.transquant_bypass_enabled_flag = true;  // SAO/deblock then honour per-CU bypass
    e.sh.slice_type = SliceType::B;
    int ns = std::max(1, (int)syn.num_slices);
    e.slices.assign((size_t)ns, SliceHeader{});
    for (int i = 0; i < ns; i++) {
        SliceHeader& s = e.slices[(size_t)i];
        s.slice_type = SliceType::B;
        if (syn.slices && i < syn.num_slices) {
            s.slice_deblocking_filter_disabled_flag = syn.slices[i].deblocking_disabled != 0;
            s.slice_beta_offset_div2 = syn.slices[i].beta_offset_div2;
            s.slice_tc_offset_div2 = syn.slices[i].tc_offset_div2;
            s.slice_loop_filter_across_slices_enabled_flag = syn.slices[i].lf_across_slices != 0;
        }
    }
    e.slice_ptrs.clear();
    for (auto& s : e.slices) e.slice_ptrs.push_back(&s);

    load_picture(e.pic, p.width, p.height, in);

    // reference pictures: RefPicList entries with their POCs (and samples when given)
    e.refs.clear();
    e.dpb.ref_pic_list0_.clear();
    e.dpb.ref_pic_list1_.clear();
    std::vector<Picture*> by_slot;
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < p.num_ref[l]; i++) {
            int slot = p.ref_slot[l][i];
            Picture* rp = nullptr;
            if (slot >= 0) {
                if ((int)by_slot.size() <= slot) by_slot.resize((size_t)slot + 1, nullptr);
                if (!by_slot[(size_t)slot]) {
                    e.refs.emplace_back(new Picture());
                    Picture* np = e.refs.back().get();
                    const uint8_t* planes = (ref_planes && slot < num_refs) ? ref_planes[slot] : nullptr;
                    load_picture(*np, p.width, p.height, planes);
                    by_slot[(size_t)slot] = np;
                }
                rp = by_slot[(size_t)slot];
                rp->poc = p.ref_poc[l][i];
            }
            RefPicListEntry ent;
            ent.pic = rp;
            (l == 0 ? e.dpb.ref_pic_list0_ : e.dpb.ref_pic_list1_).push_back(ent);
        }

    int gw = p.width / 4, gh = p.height / 4;
    int cbw = e.sps.PicWidthInMinCbsY, cbh = e.sps.PicHeightInMinCbsY;
    int mcb = e.sps.MinCbSizeY;
    e.cu_info.assign((size_t)cbw * cbh, CUInfo{});
    e.cbf.assign((size_t)gw * gh, 0);
    e.tu_log2.assign((size_t)gw * gh, 0);
    e.edge_v.assign((size_t)gw * gh, 0);
    e.edge_h.assign((size_t)gw * gh, 0);
    e.motion.assign((size_t)gw * gh, PUMotionInfo{});
    for (int gy = 0; gy < gh; gy++)
        for (int gx = 0; gx < gw; gx++) {
            uint32_t b = syn.blk[(size_t)gy * gw + gx];
            size_t i = (size_t)gy * gw + gx;
            e.cbf[i] = (b & HEVC_BLK_CBF) ? 1 : 0;
            e.tu_log2[i] = (uint8_t)((b >> HEVC_BLK_TU_SHIFT) & 0xFF);
            e.edge_v[i] = (b & HEVC_BLK_EDGE_V) ? 1 : 0;
            e.edge_h[i] = (b & HEVC_BLK_EDGE_H) ? 1 : 0;
            CUInfo& cu = e.cu_info[(size_t)(gy * 4 / mcb) * cbw + gx * 4 / mcb];
            cu.pred_mode = (b & HEVC_BLK_INTRA) ? PredMode::MODE_INTRA : PredMode::MODE_INTER;
            cu.qp_y = (int8_t)(b >> HEVC_BLK_QP_SHIFT);
            cu.is_pcm = (b & HEVC_BLK_PCM) != 0;
            cu.cu_transquant_bypass = (b & HEVC_BLK_BYPASS) != 0;
        }
    for (int i = 0; i < syn.num_pus; i++) {
        const hevc_pu_t& pu = syn.pus[i];
        PUMotionInfo mi;
        for (int l = 0; l < 2; l++) {
            mi.mv[l].x = pu.mv[l][0];
            mi.mv[l].y = pu.mv[l][1];
            mi.ref_idx[l] = pu.ref_idx[l];
            mi.pred_flag[l] = pu.ref_idx[l] >= 0;
        }
        for (int y = pu.y; y < pu.y + pu.h; y += 4)
            for (int x = pu.x; x < pu.x + pu.w; x += 4) e.motion[(size_t)(y / 4) * gw + x / 4] = mi;
    }
    int nctb = e.sps.PicSizeInCtbsY;
    e.sao.assign((size_t)nctb, DecodingContext::SaoParams{});
    e.slice_idx.assign((size_t)nctb, 0);
    for (int a = 0; a < nctb; a++) {
        if (syn.sao) {
            const hevc_sao_t& s = syn.sao[a];
            for (int c = 0; c < 3; c++) {
                e.sao[(size_t)a].sao_type_idx[c] = s.type[c];
                e.sao[(size_t)a].sao_band_position[c] = s.band_pos[c];
                e.sao[(size_t)a].sao_eo_class[c] = s.eo_class[c];
                for (int k = 0; k < 5; k++) e.sao[(size_t)a].sao_offset_val[c][k] = s.offset[c][k];
            }
        }
        if (syn.ctb_slice) e.slice_idx[(size_t)a] = syn.ctb_slice[a];
    }

    DecodingContext& c = e.ctx;
    c.sps = &e.sps;
    c.pps = &e.pps;
    c.sh = &e.slices[0];
    c.pic = &e.pic;
    c.dpb = &e.dpb;
    c.cu_info = e.cu_info.data();
    c.cu_info_stride = cbw;
    c.motion_info = e.motion.data();
    c.motion_info_stride = gw;
    c.cbf_luma_grid = e.cbf.data();
    c.log2_tu_size_grid = e.tu_log2.data();
    c.edge_flags_v = e.edge_v.data();
    c.edge_flags_h = e.edge_h.data();
    c.filter_grid_stride = gw;
    c.sao_params = e.sao.data();
    c.sao_params_stride = e.sps.PicWidthInCtbsY;
    c.sao_backup = e.sao_backup;
    c.slice_idx = e.slice_idx.data();
    c.slice_headers = e.slice_ptrs.data();
    c.num_slices = (int)e.slice_ptrs.size();
}

// Weighted-prediction switch of one PU: the reference selects explicit WP per slice
// (interpolation.cpp:392-396); the harness points the context at a PPS and a slice
// header that carry this PU's weights.
void set_pu_wp(Env& e, const hevc_pu_t& pu, const hevc_wp_t* wp_tab, PPS& pps, SliceHeader& sh) {
    pps = e.pps;
    sh = e.slices[0];
    sh.slice_type = SliceType::B;
    pps.weighted_bipred_flag = false;
    pps.weighted_pred_flag = false;
    if (pu.wp < 0) return;
    const hevc_wp_t& w = wp_tab[pu.wp];
    pps.weighted_bipred_flag = true;
    PredWeightTable& t = sh.pred_weight_table;
    t.luma_log2_weight_denom = (uint32_t)(w.log2wd[0] - 6);
    t.delta_chroma_log2_weight_denom = w.log2wd[1] - w.log2wd[0];
    int i0 = pu.ref_idx[0] >= 0 ? pu.ref_idx[0] : 0;
    int i1 = pu.ref_idx[1] >= 0 ? pu.ref_idx[1] : 0;
    t.l0[(size_t)i0].luma_weight = w.w[0][0];
    t.l0[(size_t)i0].luma_offset = w.o[0][0];
    t.l1[(size_t)i1].luma_weight = w.w[1][0];
    t.l1[(size_t)i1].luma_offset = w.o[1][0];
    for (int c = 0; c < 2; c++) {
        t.l0[(size_t)i0].chroma_weight[c] = w.w[0][c + 1];
        t.l0[(size_t)i0].chroma_offset[c] = w.o[0][c + 1];
        t.l1[(size_t)i1].chroma_weight[c] = w.w[1][c + 1];
        t.l1[(size_t)i1].chroma_offset[c] = w.o[1][c + 1];
    }
}

void mc_pu(Env& e, const hevc_pu_t& pu, const hevc_wp_t* wp_tab) {
    const auto key = pu.wp < 0 ? std::make_tuple(-1, 0, 0)
                               : std::make_tuple((int)pu.wp, pu.ref_idx[0] >= 0 ? (int)pu.ref_idx[0] : 0,
                                                 pu.ref_idx[1] >= 0 ? (int)pu.ref_idx[1] : 0);
    auto it = e.wp_forms.find(key);
    if (it == e.wp_forms.end()) {
        it = e.wp_forms.emplace(key, std::pair<PPS, SliceHeader>()).first;
        set_pu_wp(e, pu, wp_tab, it->second.first, it->second.second);
    }
    const PPS* saved_pps = e.ctx.pps;
    const SliceHeader* saved_sh = e.ctx.sh;
    e.ctx.pps = &it->second.first;
    e.ctx.sh = &it->second.second;
    MV mv0, mv1;
    mv0.x = pu.mv[0][0]; mv0.y = pu.mv[0][1];
    mv1.x = pu.mv[1][0]; mv1.y = pu.mv[1][1];
    for (int c = 0; c < 3; c++) {
        int16_t pred[64 * 64];
        perform_inter_prediction(e.ctx, pu.x, pu.y, pu.w, pu.h, c, mv0, mv1, pu.ref_idx[0], pu.ref_idx[1],
                                 pu.ref_idx[0] >= 0, pu.ref_idx[1] >= 0, pred);
        int sub = c ? 2 : 1, w = pu.w / sub, h = pu.h / sub, xc = pu.x / sub, yc = pu.y / sub;
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) e.pic.sample(c, xc + x, yc + y) = (uint16_t)pred[y * w + x];
    }
    e.ctx.pps = saved_pps;
    e.ctx.sh = saved_sh;
}

void tu_residual(Env& e, const hevc_tu_t& t, const int16_t* coeffs, int16_t* residual) {
    int n = 1 << t.log2_size;
    std::memset(residual, 0, sizeof(int16_t) * (size_t)n * n);
    if (!(t.flags & HEVC_TU_CODED)) return;
    const int16_t* lv = coeffs + t.coeff_offset;
    if (t.flags & HEVC_TU_BYPASS) {
        std::memcpy(residual, lv, sizeof(int16_t) * (size_t)n * n);
        return;
    }
    int16_t scaled[32 * 32] = {};
    int sub = t.c_idx ? 2 : 1;
    perform_dequant(e.ctx, t.x * sub, t.y * sub, t.log2_size, t.c_idx, t.qp, lv, scaled);
    perform_transform_inverse(t.log2_size, t.c_idx, (t.flags & HEVC_TU_INTRA) != 0, (t.flags & HEVC_TU_TSKIP) != 0,
                              8, scaled, residual);
}

// One TU of decode_transform_unit (coding_tree.cpp:1256-1419): prediction (intra, or
// the MC samples already in the picture), then reconstruct_block's add and clip.
void tu_recon(Env& e, const hevc_tu_t& t, const int16_t* coeffs) {
    int n = 1 << t.log2_size, c = t.c_idx, sub = c ? 2 : 1;
    if (t.flags & HEVC_TU_PCM) {   // pcm_sample values written as they are (coding_tree.cpp:1425-1469)
        const int16_t* lv = coeffs + t.coeff_offset;
        for (int y = 0; y < n; y++)
            for (int x = 0; x < n; x++)
                if (t.x + x < e.pic.width[c] && t.y + y < e.pic.height[c])
                    e.pic.sample(c, t.x + x, t.y + y) = (uint16_t)lv[y * n + x];
        return;
    }
    int16_t residual[32 * 32];
    tu_residual(e, t, coeffs, residual);
    int16_t pred[32 * 32] = {};
    if (t.flags & HEVC_TU_INTRA) {
        perform_intra_prediction(e.ctx, t.x * sub, t.y * sub, t.log2_size, c, t.intra_mode, pred);
    } else {
        for (int y = 0; y < n; y++)
            for (int x = 0; x < n; x++) pred[y * n + x] = (int16_t)e.pic.sample(c, t.x + x, t.y + y);
    }
    int pw = e.pic.width[c], ph = e.pic.height[c];
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
            if (t.x + x >= pw || t.y + y >= ph) continue;
            int v = pred[y * n + x] + residual[y * n + x];
            e.pic.sample(c, t.x + x, t.y + y) = (uint16_t)Clip3(0, 255, v);
        }
}

}  // namespace

extern "C" {

// Independent blocks at (0,0) of a one-CU grid whose prediction mode follows each
// block's HEVC_TU_INTRA flag (perform_dequant reads it through cu_at with scaling lists).
int ref_residual_blocks_scaled(const hevc_scaling_t* sl, const hevc_tu_t* tus, int32_t num_tus,
                               const int16_t* coeffs, const uint8_t* pred, uint8_t* out) {
    Env e;
    init_sps(e.sps, 64, 64, 6, 3, 0, 0, 0, 0);
    set_scaling(e.sps, sl);
    e.cu_info.assign(1, CUInfo{});
    e.ctx.sps = &e.sps;
    e.ctx.pps = &e.pps;
    e.ctx.cu_info = e.cu_info.data();
    e.ctx.cu_info_stride = 1;
    for (int i = 0; i < num_tus; i++) {
        const hevc_tu_t& t = tus[i];
        int n = 1 << t.log2_size;
        e.cu_info[0].pred_mode = (t.flags & HEVC_TU_INTRA) ? PredMode::MODE_INTRA : PredMode::MODE_INTER;
        int16_t scaled[32 * 32] = {}, residual[32 * 32] = {};
        perform_dequant(e.ctx, 0, 0, t.log2_size, t.c_idx, t.qp, coeffs + t.coeff_offset, scaled);
        perform_transform_inverse(t.log2_size, t.c_idx, (t.flags & HEVC_TU_INTRA) != 0,
                                  (t.flags & HEVC_TU_TSKIP) != 0, 8, scaled, residual);
        for (int k = 0; k < n * n; k++) {
            int v = pred[t.coeff_offset + k] + residual[k];
            out[t.coeff_offset + k] = (uint8_t)Clip3(0, 255, v);
        }
    }
    return 0;
}

int ref_residual_blocks(const hevc_tu_t* tus, int32_t num_tus, const int16_t* coeffs, const uint8_t* pred,
                        uint8_t* out) {
    return ref_residual_blocks_scaled(nullptr, tus, num_tus, coeffs, pred, out);
}

int ref_inter_pred(const hevc_pic_params_t* pp, const hevc_pu_t* pus, int32_t num_pus, const hevc_wp_t* wp,
                   int32_t num_wp, const uint8_t* const* refs, int32_t num_refs, uint8_t* out) {
    (void)num_wp;
    hevc_picture_syntax_t syn;
    std::memset(&syn, 0, sizeof(syn));
    syn.params = *pp;
    std::vector<uint32_t> blk((size_t)(pp->width / 4) * (pp->height / 4), 0);
    syn.blk = blk.data();
    Env e;
    setup(e, syn, nullptr, refs, num_refs);
    for (int i = 0; i < num_pus; i++) mc_pu(e, pus[i], wp);
    store_picture(e.pic, out);
    return 0;
}

int ref_loop_filter(const hevc_picture_syntax_t* syn, const uint8_t* in, uint8_t* out, int do_deblock,
                    int do_sao) {
    Env e;
    setup(e, *syn, in, nullptr, 0);
    if (do_deblock) apply_deblocking(e.ctx);
    if (do_sao) apply_sao(e.ctx);
    store_picture(e.pic, out);
    return 0;
}

int ref_intra_recon(const hevc_picture_syntax_t* syn, const uint8_t* in, uint8_t* out) {
    Env e;
    setup(e, *syn, in, nullptr, 0);
    for (int i = 0; i < syn->num_tus; i++)
        if (syn->tus[i].flags & HEVC_TU_INTRA) tu_recon(e, syn->tus[i], syn->coeffs);
    store_picture(e.pic, out);
    return 0;
}

// Whole picture in the reference's own decode order: CU by CU, MC of its PUs first,
// then its transform units in decode order, then deblocking and SAO over the picture.
int ref_reconstruct_picture(const hevcsynth_picture_t* pic, const uint8_t* const* refs, int32_t num_refs,
                            uint8_t* out) {
    const hevc_picture_syntax_t& syn = pic->syn;
    Env e;
    setup(e, syn, nullptr, refs, num_refs);
    for (int i = 0; i < pic->num_cus; i++) {
        const hevcsynth_cu_t& cu = pic->cus[i];
        for (int k = 0; k < cu.num_pu; k++) mc_pu(e, syn.pus[cu.first_pu + k], syn.wp);
        for (int k = 0; k < cu.num_tu; k++) tu_recon(e, syn.tus[cu.first_tu + k], syn.coeffs);
    }
    apply_deblocking(e.ctx);
    apply_sao(e.ctx);
    store_picture(e.pic, out);
    return 0;
}

}  // extern "C"
