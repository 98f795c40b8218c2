// recorder.cpp — privaloops/hevc.js decodes a real stream; every picture is recorded as the
// records of include/hevcgpu.h, and the oracle reconstructs it from them.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `record`) into
// oracle/_ref/hevc-record, against the reference's own objects in oracle/_ref/libhevcdec.so.
//
// The reference's hooks of the reconstruction path — perform_dequant and
// perform_transform_inverse (src/decoding/transform.cpp:293, :374), perform_intra_prediction
// (src/decoding/intra_prediction.cpp:428), perform_inter_prediction
// (src/decoding/interpolation.cpp:306), apply_deblocking (src/filters/deblocking.cpp:357) and
// apply_sao (src/filters/sao.cpp:20) — are defined here as well.  The reference's coding tree
// (in the shared library) calls them through the dynamic linker, so these definitions run
// first; each records its arguments and calls the reference's own definition (dlsym
// RTLD_NEXT), so the stream decodes exactly as it does without them.  This is the recorder
// the integration plan describes, run inside the unmodified reference.
//
// Per picture, after the reference's SAO, the oracle (hevc_oracle.c) reconstructs the
// picture from the records and from its own earlier outputs as reference pictures, and the
// result is compared with the reference's picture.  One line per picture:
//   picture <n> poc <p>: match (<TUs>, <PUs>) fnv <FNV-1a 64 of the reference's I420 picture>
//                      | mismatch <samples> | unsupported (<why>)
// With a second argument the records of every picture the oracle matched are written to that
// file (with a third argument "--all", those of unsupported pictures too, as long as no
// picture mismatched: the syntax the reference parsed, for checking a stream's parse), with
// the references as decode indices of earlier pictures:
//   "HREC" u32 version (1), then per picture: hevc_pic_params_t (ref_slot entries: decode
//   index of the referenced picture), i32 counts of TUs, levels, PUs, WP rows and slices,
//   u8 has_scaling, u8 has_tiles, 2 pad bytes, then the arrays: TUs, levels, PUs, WP rows,
//   the blk grid, SAO per CTB, slice index per CTB, tile id per CTB (when has_tiles),
//   slices, scaling lists (when has_scaling).
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common/picture.h"
#include "common/types.h"
#include "decoding/coding_tree.h"
#include "syntax/pps.h"
#include "syntax/slice_header.h"
#include "syntax/sps.h"
// the DPB's reference lists are private; the recorder reads them
#define private public
#include "decoding/dpb.h"
#undef private
#include "wasm/hevc_api.h"

#include "../include/hevcgpu.h"

extern "C" int oracle_reconstruct_picture(const hevc_picture_syntax_t* syn, const uint8_t* const* refs,
                                          int32_t num_refs, uint8_t* out);

using namespace hevc;

namespace {

template <typename F>
F real(const char* name) {
    void* p = dlsym(RTLD_NEXT, name);
    if (!p) {
        std::fprintf(stderr, "recorder: %s not found\n", name);
        std::exit(2);
    }
    return reinterpret_cast<F>(p);
}

struct Picture8 {   // an 8-bit I420 picture
    int w = 0, h = 0;
    std::vector<uint8_t> s;
};

struct Recording {
    std::mutex mu;
    std::vector<hevc_tu_t> tus;
    std::vector<int16_t> coeffs;
    std::vector<hevc_pu_t> pus;
    std::vector<hevc_wp_t> wp;
    std::vector<const Picture*> pu_ref[2];   // per PU: the reference picture of each list
    std::string unsupported;
    std::map<const Picture*, Picture8> ours;  // the oracle's output for each reference Picture object
    std::map<const Picture*, int> index_of;   // decode index of the picture each Picture object holds
    FILE* dump = nullptr;
    bool dump_all = false;   // also write the records of unsupported pictures
    // the picture's records, built at apply_deblocking
    hevc_picture_syntax_t syn{};
    std::vector<uint32_t> blk;
    std::vector<hevc_sao_t> sao;
    std::vector<uint8_t> ctb_slice;
    std::vector<uint16_t> ctb_tile;
    std::vector<hevc_slice_t> slices;
    hevc_scaling_t scaling{};
    std::vector<const Picture*> refs;
    int pictures = 0, matched = 0, mismatched = 0, skipped = 0;
} R;

struct Pending {   // the coded TU between its dequantisation and its prediction
    bool active = false;
    hevc_tu_t t{};
    std::vector<int16_t> lv;
};
thread_local Pending P;

void append_tu(hevc_tu_t t, const std::vector<int16_t>& lv) {
    std::lock_guard<std::mutex> g(R.mu);
    if (t.flags & HEVC_TU_CODED) {
        t.coeff_offset = (uint32_t)R.coeffs.size();
        R.coeffs.insert(R.coeffs.end(), lv.begin(), lv.end());
    }
    R.tus.push_back(t);
}

void note_unsupported(const std::string& why) {
    std::lock_guard<std::mutex> g(R.mu);
    if (R.unsupported.empty()) R.unsupported = why;
}

}  // namespace

namespace hevc {

void perform_dequant(DecodingContext& ctx, int x0, int y0, int log2, int cIdx, int qp, const int16_t* coefficients,
                     int16_t* scaled) {
    static auto f = real<decltype(&perform_dequant)>("_ZN4hevc15perform_dequantERNS_15DecodingContextEiiiiiPKsPs");
    const int sub = cIdx ? 2 : 1, n = 1 << log2;
    P.active = true;
    P.t = hevc_tu_t{};
    P.t.x = (uint16_t)(x0 / sub);
    P.t.y = (uint16_t)(y0 / sub);
    P.t.log2_size = (uint8_t)log2;
    P.t.c_idx = (uint8_t)cIdx;
    P.t.qp = (uint8_t)qp;
    P.t.flags = HEVC_TU_CODED;
    P.lv.assign(coefficients, coefficients + n * n);
    f(ctx, x0, y0, log2, cIdx, qp, coefficients, scaled);
}

void perform_transform_inverse(int log2, int cIdx, bool is_intra, bool transform_skip, int bit_depth,
                               const int16_t* scaled, int16_t* residual) {
    static auto f = real<decltype(&perform_transform_inverse)>("_ZN4hevc25perform_transform_inverseEiibbiPKsPs");
    f(log2, cIdx, is_intra, transform_skip, bit_depth, scaled, residual);
    if (!P.active) return;
    if (transform_skip) P.t.flags |= HEVC_TU_TSKIP;
    if (!is_intra) {   // an inter TU: complete (its prediction is the PU's)
        append_tu(P.t, P.lv);
        P.active = false;
    }
}

void perform_intra_prediction(DecodingContext& ctx, int x0, int y0, int log2, int cIdx, int mode, int16_t* pred) {
    static auto f = real<decltype(&perform_intra_prediction)>("_ZN4hevc24perform_intra_predictionERNS_15DecodingContextEiiiiiPs");
    f(ctx, x0, y0, log2, cIdx, mode, pred);
    const int sub = cIdx ? 2 : 1;
    hevc_tu_t t{};
    std::vector<int16_t> lv;
    if (P.active && P.t.c_idx == cIdx && P.t.x == x0 / sub && P.t.y == y0 / sub && P.t.log2_size == log2) {
        t = P.t;
        lv.swap(P.lv);
        P.active = false;
    } else {   // an intra TU without levels
        t.x = (uint16_t)(x0 / sub);
        t.y = (uint16_t)(y0 / sub);
        t.log2_size = (uint8_t)log2;
        t.c_idx = (uint8_t)cIdx;
    }
    t.flags |= HEVC_TU_INTRA;
    t.intra_mode = (uint8_t)mode;
    append_tu(t, lv);
}

void perform_inter_prediction(DecodingContext& ctx, int xPb, int yPb, int w, int h, int cIdx, const MV& mv0,
                              const MV& mv1, int ref0, int ref1, bool pf0, bool pf1, int16_t* pred) {
    static auto f = real<decltype(&perform_inter_prediction)>(
        "_ZN4hevc24perform_inter_predictionERNS_15DecodingContextEiiiiiRKNS_2MVES4_iibbPs");
    f(ctx, xPb, yPb, w, h, cIdx, mv0, mv1, ref0, ref1, pf0, pf1, pred);
    if (cIdx != 0) return;
    hevc_pu_t u{};
    u.x = (uint16_t)xPb;
    u.y = (uint16_t)yPb;
    u.w = (uint8_t)w;
    u.h = (uint8_t)h;
    u.ref_idx[0] = (int8_t)(pf0 ? ref0 : -1);
    u.ref_idx[1] = (int8_t)(pf1 ? ref1 : -1);
    u.mv[0][0] = (int16_t)mv0.x;
    u.mv[0][1] = (int16_t)mv0.y;
    u.mv[1][0] = (int16_t)mv1.x;
    u.mv[1][1] = (int16_t)mv1.y;
    u.wp = -1;
    // explicit weighted prediction of the PU's slice (interpolation.cpp:392-400, :246-300)
    const SliceHeader& sh = *ctx.sh;
    const bool wpf = (sh.slice_type == SliceType::P && ctx.pps->weighted_pred_flag) ||
                     (sh.slice_type == SliceType::B && ctx.pps->weighted_bipred_flag);
    hevc_wp_t wt{};
    if (wpf) {
        const PredWeightTable& t = sh.pred_weight_table;
        wt.log2wd[0] = (int16_t)(t.luma_log2_weight_denom + 6);
        wt.log2wd[1] = (int16_t)((int)t.luma_log2_weight_denom + t.delta_chroma_log2_weight_denom + 6);
        const PredWeightTable::RefWeight* rw[2] = {&t.l0[(size_t)(ref0 >= 0 ? ref0 : 0)],
                                                   &t.l1[(size_t)(ref1 >= 0 ? ref1 : 0)]};
        for (int l = 0; l < 2; l++) {
            wt.w[l][0] = rw[l]->luma_weight;
            wt.o[l][0] = rw[l]->luma_offset;
            for (int c = 0; c < 2; c++) {
                wt.w[l][c + 1] = rw[l]->chroma_weight[c];
                wt.o[l][c + 1] = rw[l]->chroma_offset[c];
            }
        }
    }
    const Picture* rp[2] = {pf0 ? ctx.dpb->ref_pic_list0(ref0) : nullptr, pf1 ? ctx.dpb->ref_pic_list1(ref1) : nullptr};
    std::lock_guard<std::mutex> g(R.mu);
    if (wpf) {
        u.wp = (int16_t)R.wp.size();
        R.wp.push_back(wt);
    }
    R.pus.push_back(u);
    R.pu_ref[0].push_back(rp[0]);
    R.pu_ref[1].push_back(rp[1]);
}

// A slice segment's data (coding_tree.cpp:536).  With WPP the reference decodes CTU rows on
// its thread pool, each row waiting for the second CTU of the row above and every row from
// column 0 to the picture's end (coding_tree.cpp:404-533); a picture one CTU wide has no
// second CTU and the rows would wait for good, and a picture of several slice segments is
// decoded from the wrong substreams.  Such pictures take the reference's own sequential
// path (no thread pool).  The drop-in does the same (dropin/hooks.cpp).
bool decode_slice_segment_data(DecodingContext& ctx, BitstreamReader& bs, const std::vector<size_t>& epb,
                               size_t header_size) {
    static auto f = real<bool (*)(DecodingContext&, BitstreamReader&, const std::vector<size_t>&, size_t)>(
        "_ZN4hevc25decode_slice_segment_dataERNS_15DecodingContextERNS_15BitstreamReaderERKSt6vectorImSaImEEm");
    ThreadPool* pool = ctx.thread_pool;
    if (pool && ctx.pps && ctx.pps->entropy_coding_sync_enabled_flag && ctx.sps &&
        (ctx.sps->PicWidthInCtbsY == 1 || ctx.num_slices > 1)) {
        ctx.thread_pool = nullptr;
        const bool ok = f(ctx, bs, epb, header_size);
        ctx.thread_pool = pool;
        return ok;
    }
    return f(ctx, bs, epb, header_size);
}

// The picture's records from the context the reference's filters read
// (decoder.cpp:117-185 fills it; the harness in ref_harness.cpp does the inverse).
void apply_deblocking(DecodingContext& ctx) {
    static auto f = real<decltype(&apply_deblocking)>("_ZN4hevc16apply_deblockingERNS_15DecodingContextE");
    const SPS& sps = *ctx.sps;
    const PPS& pps = *ctx.pps;
    const int W = (int)sps.pic_width_in_luma_samples, H = (int)sps.pic_height_in_luma_samples;
    const int gw = W / 4, gh = H / 4, nctb = sps.PicSizeInCtbsY;
    if (sps.BitDepthY != 8 || sps.BitDepthC != 8) note_unsupported("bit depth above 8");
    if (sps.chroma_format_idc != 1) note_unsupported("not 4:2:0");
    R.blk.assign((size_t)gw * gh, 0u);
    bool pcm_or_bypass = false;
    for (int gy = 0; gy < gh; gy++)
        for (int gx = 0; gx < gw; gx++) {
            const size_t g = (size_t)gy * ctx.filter_grid_stride + gx;
            const CUInfo& cu = ctx.cu_at(gx * 4, gy * 4);
            uint32_t b = (ctx.edge_flags_v[g] ? HEVC_BLK_EDGE_V : 0u) | (ctx.edge_flags_h[g] ? HEVC_BLK_EDGE_H : 0u) |
                         (ctx.cbf_luma_grid[g] ? HEVC_BLK_CBF : 0u) |
                         (cu.pred_mode == PredMode::MODE_INTRA ? HEVC_BLK_INTRA : 0u) |
                         (cu.is_pcm ? HEVC_BLK_PCM : 0u) | (cu.cu_transquant_bypass ? HEVC_BLK_BYPASS : 0u) |
                         ((uint32_t)ctx.log2_tu_size_grid[g] << HEVC_BLK_TU_SHIFT) |
                         ((uint32_t)(uint8_t)cu.qp_y << HEVC_BLK_QP_SHIFT);
            pcm_or_bypass |= cu.is_pcm || cu.cu_transquant_bypass;
            R.blk[(size_t)gy * gw + gx] = b;
        }
    if (pcm_or_bypass) note_unsupported("PCM or transquant-bypass CUs (the recorder sees no levels for them)");
    R.sao.assign((size_t)nctb, hevc_sao_t{});
    for (int a = 0; a < nctb; a++) {
        const auto& s = ctx.sao_params[a];
        for (int c = 0; c < 3; c++) {
            R.sao[(size_t)a].type[c] = (uint8_t)s.sao_type_idx[c];
            R.sao[(size_t)a].band_pos[c] = (uint8_t)s.sao_band_position[c];
            R.sao[(size_t)a].eo_class[c] = (uint8_t)s.sao_eo_class[c];
            for (int k = 0; k < 5; k++) R.sao[(size_t)a].offset[c][k] = (int8_t)s.sao_offset_val[c][k];
        }
    }
    R.ctb_slice.assign(ctx.slice_idx, ctx.slice_idx + nctb);
    R.slices.clear();
    for (int k = 0; k < ctx.num_slices; k++) {
        const SliceHeader& s = *ctx.slice_headers[k];
        R.slices.push_back(hevc_slice_t{(int8_t)s.slice_beta_offset_div2, (int8_t)s.slice_tc_offset_div2,
                                        (uint8_t)s.slice_deblocking_filter_disabled_flag,
                                        (uint8_t)s.slice_loop_filter_across_slices_enabled_flag});
    }
    R.ctb_tile.assign((size_t)nctb, 0);
    if (!pps.TileId.empty())
        for (int a = 0; a < nctb; a++) R.ctb_tile[(size_t)a] = (uint16_t)pps.TileId[(size_t)pps.CtbAddrRsToTs[(size_t)a]];

    hevc_picture_syntax_t& syn = R.syn;
    std::memset(&syn, 0, sizeof(syn));
    hevc_pic_params_t& p = syn.params;
    p.width = W;
    p.height = H;
    p.bit_depth = 8;
    p.log2_ctb = sps.CtbLog2SizeY;
    p.log2_min_cb = (int)sps.log2_min_luma_coding_block_size_minus3 + 3;
    p.log2_min_tb = (int)sps.log2_min_luma_transform_block_size_minus2 + 2;
    p.strong_intra_smoothing = sps.strong_intra_smoothing_enabled_flag;
    p.intra_smoothing_disabled = sps.intra_smoothing_disabled_flag;
    p.pcm_loop_filter_disabled = sps.pcm_loop_filter_disabled_flag;
    p.sao_enabled = sps.sample_adaptive_offset_enabled_flag;
    p.cb_qp_offset = pps.pps_cb_qp_offset;
    p.cr_qp_offset = pps.pps_cr_qp_offset;
    p.tiles_enabled = pps.tiles_enabled_flag;
    p.loop_filter_across_tiles = pps.loop_filter_across_tiles_enabled_flag;
    // reference lists as the filters see them at this point (deblocking.cpp:183-193); the
    // PUs' pictures must be these
    R.refs.clear();
    auto slot_of = [&](const Picture* pic) {
        for (size_t k = 0; k < R.refs.size(); k++)
            if (R.refs[k] == pic) return (int)k;
        R.refs.push_back(pic);
        return (int)R.refs.size() - 1;
    };
    const int n_list[2] = {ctx.dpb->num_ref_list0(), ctx.dpb->num_ref_list1()};
    for (int l = 0; l < 2; l++) {
        p.num_ref[l] = std::min(n_list[l], 16);
        for (int i = 0; i < 16; i++) {
            p.ref_poc[l][i] = -999999;
            p.ref_slot[l][i] = -1;
        }
        for (int i = 0; i < p.num_ref[l]; i++) {
            const Picture* rp = l == 0 ? ctx.dpb->ref_pic_list0(i) : ctx.dpb->ref_pic_list1(i);
            if (!rp) continue;
            p.ref_poc[l][i] = rp->poc;
            p.ref_slot[l][i] = slot_of(rp);
        }
    }
    for (size_t k = 0; k < R.pus.size(); k++)
        for (int l = 0; l < 2; l++) {
            const int idx = R.pus[k].ref_idx[l];
            if (idx < 0) continue;
            const Picture* want = idx < p.num_ref[l] ? (l == 0 ? ctx.dpb->ref_pic_list0(idx) : ctx.dpb->ref_pic_list1(idx))
                                                     : nullptr;
            if (want != R.pu_ref[l][k]) note_unsupported("reference lists that differ between slices");
        }
    if (sps.scaling_list_enabled_flag) {
        const ScalingListData& sl = pps.pps_scaling_list_data_present_flag ? pps.scaling_list_data : sps.scaling_list_data;
        for (int sz = 0; sz < 4; sz++)
            for (int m = 0; m < 6; m++) std::memcpy(R.scaling.list[sz][m], sl.scaling_list[(size_t)sz][(size_t)m].data(), 64);
        for (int i = 0; i < 2; i++)
            for (int m = 0; m < 6; m++) R.scaling.dc[i][m] = sl.scaling_list_dc[(size_t)i][(size_t)m];
        syn.scaling = &R.scaling;
    }
    syn.num_tus = (int32_t)R.tus.size();
    syn.tus = R.tus.data();
    syn.num_coeffs = R.coeffs.size();
    syn.coeffs = R.coeffs.data();
    syn.num_pus = (int32_t)R.pus.size();
    syn.pus = R.pus.data();
    syn.num_wp = (int32_t)R.wp.size();
    syn.wp = R.wp.data();
    syn.blk = R.blk.data();
    syn.sao = R.sao.data();
    syn.ctb_slice = R.ctb_slice.data();
    syn.ctb_tile = pps.TileId.empty() ? nullptr : R.ctb_tile.data();
    syn.num_slices = (int32_t)R.slices.size();
    syn.slices = R.slices.data();
    f(ctx);
}

// After the reference's SAO the picture is final: reconstruct it with the oracle from the
// records and compare.
void apply_sao(DecodingContext& ctx) {
    static auto f = real<decltype(&apply_sao)>("_ZN4hevc9apply_saoERNS_15DecodingContextE");
    f(ctx);
    const Picture& pic = *ctx.pic;
    const int W = R.syn.params.width, H = R.syn.params.height;
    const int n = R.pictures++;
    std::string why = R.unsupported;
    std::vector<const uint8_t*> refs;
    for (const Picture* rp : R.refs) {
        auto it = R.ours.find(rp);
        if (it == R.ours.end()) {
            if (why.empty()) why = "a reference picture the oracle has not reconstructed";
            refs.push_back(nullptr);
        } else {
            refs.push_back(it->second.s.data());
        }
    }
    Picture8 out;
    out.w = W;
    out.h = H;
    out.s.assign((size_t)W * H * 3 / 2, 0);
    if (why.empty() && oracle_reconstruct_picture(&R.syn, refs.data(), (int32_t)refs.size(), out.s.data()) != 0)
        why = "the oracle refused the records";
    if (!why.empty()) {
        std::printf("picture %d poc %d: unsupported (%s)\n", n, pic.poc, why.c_str());
        R.skipped++;
    } else {
        size_t diff = 0, at = 0;
        for (int c = 0; c < 3; c++) {
            const int w = c ? W / 2 : W, h = c ? H / 2 : H;
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++, at++) diff += out.s[at] != (uint8_t)pic.planes[c][(size_t)y * pic.stride[c] + x];
        }
        if (diff == 0) {
            uint64_t fnv = 1469598103934665603ull;   // equal to the reference's samples here
            for (uint8_t v : out.s) fnv = (fnv ^ v) * 1099511628211ull;
            std::printf("picture %d poc %d: match (%d TUs, %d PUs) fnv %016llx\n", n, pic.poc, R.syn.num_tus,
                        R.syn.num_pus, (unsigned long long)fnv);
            R.matched++;
        } else {
            std::printf("picture %d poc %d: mismatch %zu samples\n", n, pic.poc, diff);
            R.mismatched++;
        }
    }
    if (R.dump && R.mismatched == 0 && (why.empty() || R.dump_all)) {   // the records of a matched picture
        hevc_picture_syntax_t s = R.syn;
        for (int l = 0; l < 2; l++)
            for (int i = 0; i < s.params.num_ref[l]; i++)
                if (s.params.ref_slot[l][i] >= 0) s.params.ref_slot[l][i] = R.index_of[R.refs[(size_t)s.params.ref_slot[l][i]]];
        const int32_t counts[5] = {s.num_tus, (int32_t)s.num_coeffs, s.num_pus, s.num_wp, s.num_slices};
        const uint8_t flags[4] = {(uint8_t)(s.scaling != nullptr), (uint8_t)(s.ctb_tile != nullptr), 0, 0};
        const int ctb = 1 << s.params.log2_ctb, nctb = ((W + ctb - 1) / ctb) * ((H + ctb - 1) / ctb);
        std::fwrite(&s.params, sizeof(s.params), 1, R.dump);
        std::fwrite(counts, sizeof(counts), 1, R.dump);
        std::fwrite(flags, sizeof(flags), 1, R.dump);
        std::fwrite(s.tus, sizeof(hevc_tu_t), (size_t)s.num_tus, R.dump);
        std::fwrite(s.coeffs, sizeof(int16_t), (size_t)s.num_coeffs, R.dump);
        std::fwrite(s.pus, sizeof(hevc_pu_t), (size_t)s.num_pus, R.dump);
        std::fwrite(s.wp, sizeof(hevc_wp_t), (size_t)s.num_wp, R.dump);
        std::fwrite(s.blk, sizeof(uint32_t), (size_t)(W / 4) * (H / 4), R.dump);
        std::fwrite(s.sao, sizeof(hevc_sao_t), (size_t)nctb, R.dump);
        std::fwrite(s.ctb_slice, 1, (size_t)nctb, R.dump);
        if (s.ctb_tile) std::fwrite(s.ctb_tile, sizeof(uint16_t), (size_t)nctb, R.dump);
        std::fwrite(s.slices, sizeof(hevc_slice_t), (size_t)s.num_slices, R.dump);
        if (s.scaling) std::fwrite(s.scaling, sizeof(hevc_scaling_t), 1, R.dump);
    }
    R.index_of[&pic] = n;
    R.ours[&pic] = std::move(out);
    R.tus.clear();
    R.coeffs.clear();
    R.pus.clear();
    R.wp.clear();
    R.pu_ref[0].clear();
    R.pu_ref[1].clear();
    R.unsupported.clear();
}

}  // namespace hevc

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: hevc-record <stream.265> [records.hrec [--all]]\n");
        return 2;
    }
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp) {
        std::fprintf(stderr, "hevc-record: cannot open %s\n", argv[1]);
        return 2;
    }
    std::vector<uint8_t> data;
    uint8_t buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), fp)) > 0) data.insert(data.end(), buf, buf + got);
    std::fclose(fp);
    if (argc > 3 && std::strcmp(argv[3], "--all") == 0) R.dump_all = true;
    if (argc > 2) {
        R.dump = std::fopen(argv[2], "wb");
        if (!R.dump) {
            std::fprintf(stderr, "hevc-record: cannot write %s\n", argv[2]);
            return 2;
        }
        const uint32_t version = 1;
        std::fwrite("HREC", 1, 4, R.dump);
        std::fwrite(&version, 4, 1, R.dump);
    }
    HEVCDecoder* dec = hevc_decoder_create();
    const int rc = hevc_decoder_decode(dec, data.data(), data.size());
    hevc_decoder_flush(dec);
    hevc_decoder_destroy(dec);
    if (R.dump) std::fclose(R.dump);
    std::printf("pictures %d matched %d mismatched %d unsupported %d decode_rc %d\n", R.pictures, R.matched,
                R.mismatched, R.skipped, rc);
    return R.mismatched ? 1 : 0;
}
