// bitgen.cpp — seeded generator of random-syntax HEVC bitstreams (bitgen.h).
//
// Rec. ITU-T H.265 (v1, Main profile), restated: the NAL unit and parameter-set syntax of
// clause 7.3, the coding-tree syntax of 7.3.8, and the CABAC encoder of 9.3 (context
// initialisation 9.3.2.2, binarisations 9.3.3, context selection 9.3.4.2, arithmetic
// encoding 9.3.4.3).  The reference decoder's counterparts are src/decoding/cabac.cpp:38
// (the decoding engine), syntax_elements.cpp (binarisations and context selection) and
// residual_coding.cpp:175 (residual_coding()).
#include "bitgen.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

namespace {

// ---- bits and NAL units -----------------------------------------------------------------
struct Bits {
    std::vector<uint8_t> buf;
    uint32_t cur = 0;
    int n = 0;
    void bit(int b) {
        cur = (cur << 1) | (uint32_t)(b & 1);
        if (++n == 8) {
            buf.push_back((uint8_t)cur);
            cur = 0;
            n = 0;
        }
    }
    void put(uint32_t v, int bits) {
        for (int i = bits - 1; i >= 0; i--) bit((int)((v >> i) & 1u));
    }
    void ue(uint32_t v) {   // Exp-Golomb, 9.2
        const uint64_t x = (uint64_t)v + 1;
        int len = 0;
        while ((x >> (len + 1)) != 0) len++;
        put(0, len);
        for (int i = len; i >= 0; i--) bit((int)((x >> i) & 1u));
    }
    void se(int32_t v) { ue(v <= 0 ? (uint32_t)(-2 * (int64_t)v) : (uint32_t)(2 * (int64_t)v - 1)); }
    void align_zero() {
        while (n) bit(0);
    }
    void trailing() {   // rbsp_trailing_bits
        bit(1);
        align_zero();
    }
};

// Annex B: start code, NAL unit header (nuh_layer_id 0, TemporalId 0), emulation prevention.
void nal(std::vector<uint8_t>& out, int type, const std::vector<uint8_t>& rbsp) {
    const uint8_t sc[4] = {0, 0, 0, 1};
    out.insert(out.end(), sc, sc + 4);
    out.push_back((uint8_t)(type << 1));
    out.push_back(1);
    int zeros = 0;
    for (uint8_t b : rbsp) {
        if (zeros >= 2 && b <= 3) {
            out.push_back(3);
            zeros = 0;
        }
        out.push_back(b);
        zeros = b == 0 ? zeros + 1 : 0;
    }
}

// ---- CABAC encoder (9.3.4.3) ------------------------------------------------------------
const uint8_t kRangeLps[64][4] = {
    {128, 176, 208, 240}, {128, 167, 197, 227}, {128, 158, 187, 216}, {123, 150, 178, 205}, {116, 142, 169, 195},
    {111, 135, 160, 185}, {105, 128, 152, 175}, {100, 122, 144, 166}, {95, 116, 137, 158},  {90, 110, 130, 150},
    {85, 104, 123, 142},  {81, 99, 117, 135},   {77, 94, 111, 128},   {73, 89, 105, 122},   {69, 85, 100, 116},
    {66, 80, 95, 110},    {62, 76, 90, 104},    {59, 72, 86, 99},     {56, 69, 81, 94},     {53, 65, 77, 89},
    {51, 62, 73, 85},     {48, 59, 69, 80},     {46, 56, 66, 76},     {43, 53, 63, 72},     {41, 50, 59, 69},
    {39, 48, 56, 65},     {37, 45, 54, 62},     {35, 43, 51, 59},     {33, 41, 48, 56},     {32, 39, 46, 53},
    {30, 37, 43, 50},     {29, 35, 41, 48},     {27, 33, 39, 45},     {26, 31, 37, 43},     {24, 30, 35, 41},
    {23, 28, 33, 39},     {22, 27, 32, 37},     {21, 26, 30, 35},     {20, 24, 29, 33},     {19, 23, 27, 31},
    {18, 22, 26, 30},     {17, 21, 25, 28},     {16, 20, 23, 27},     {15, 19, 22, 25},     {14, 18, 21, 24},
    {14, 17, 20, 23},     {13, 16, 19, 22},     {12, 15, 18, 21},     {12, 14, 17, 20},     {11, 14, 16, 19},
    {11, 13, 15, 18},     {10, 12, 15, 17},     {10, 12, 14, 16},     {9, 11, 13, 15},      {9, 11, 12, 14},
    {8, 10, 12, 14},      {8, 9, 11, 13},       {7, 9, 11, 12},       {7, 9, 10, 12},       {7, 8, 10, 11},
    {6, 8, 9, 11},        {6, 7, 9, 10},        {6, 7, 8, 9},         {2, 2, 2, 2}};
const uint8_t kNextLps[64] = {0,  0,  1,  2,  2,  4,  4,  5,  6,  7,  8,  9,  9,  11, 11, 12, 13, 13, 15, 15, 16, 16,
                              18, 18, 19, 19, 21, 21, 22, 22, 23, 24, 24, 25, 26, 26, 27, 27, 28, 29, 29, 30, 30, 30,
                              31, 32, 32, 33, 33, 33, 34, 34, 35, 35, 35, 36, 36, 36, 37, 37, 37, 38, 38, 63};

struct Ctx {
    uint8_t state = 0, mps = 0;
    void init(int init_value, int qp) {   // 9.3.2.2
        const int slope = init_value >> 4, offset = init_value & 15;
        const int m = slope * 5 - 45, n = (offset << 3) - 16;
        const int pre = std::min(126, std::max(1, ((m * std::min(51, std::max(0, qp))) >> 4) + n));
        mps = pre <= 63 ? 0 : 1;
        state = (uint8_t)(mps ? pre - 64 : 63 - pre);
    }
};

struct Cabac {
    Bits* out = nullptr;
    uint32_t low = 0, range = 510;
    int outstanding = 0;
    bool first = true;
    void start(Bits* b) {
        out = b;
        low = 0;
        range = 510;
        outstanding = 0;
        first = true;
    }
    void put_bit(int b) {
        if (first) first = false;
        else out->bit(b);
        for (; outstanding > 0; outstanding--) out->bit(1 - b);
    }
    void renorm() {
        while (range < 256) {
            if (low < 256) put_bit(0);
            else if (low >= 512) {
                low -= 512;
                put_bit(1);
            } else {
                low -= 256;
                outstanding++;
            }
            range <<= 1;
            low <<= 1;
        }
    }
    void decision(Ctx& c, int bin) {
        const uint32_t lps = kRangeLps[c.state][(range >> 6) & 3];
        range -= lps;
        if (bin != c.mps) {
            low += range;
            range = lps;
            if (c.state == 0) c.mps = (uint8_t)(1 - c.mps);
            c.state = kNextLps[c.state];
        } else if (c.state < 62) {
            c.state++;
        }
        renorm();
    }
    void bypass(int bin) {
        low <<= 1;
        if (bin) low += range;
        if (low >= 1024) {
            put_bit(1);
            low -= 1024;
        } else if (low < 512) {
            put_bit(0);
        } else {
            low -= 512;
            outstanding++;
        }
    }
    void bypass_bits(uint32_t v, int bits) {
        for (int i = bits - 1; i >= 0; i--) bypass((int)((v >> i) & 1u));
    }
    // terminate bin; after a 1 the arithmetic code is flushed, its last bit being the
    // rbsp_stop_one_bit of the slice data (9.3.4.3.5)
    void terminate(int bin) {
        range -= 2;
        if (bin) {
            low += range;
            range = 2;
            renorm();
            put_bit((int)((low >> 9) & 1u));
            out->put(((low >> 7) & 3u) | 1u, 2);
        } else {
            renorm();
        }
    }
};

// Context initialisation values of I slices (initType 0), 9.3.2.2 tables 9-5 .. 9-37.
const uint8_t kInitSaoMerge = 153;
const uint8_t kInitSaoType = 200;
const uint8_t kInitSplitCu[3] = {139, 141, 157};
const uint8_t kInitPartMode = 184;
const uint8_t kInitPrevIntraLuma = 184;
const uint8_t kInitIntraChroma = 63;
const uint8_t kInitSplitTransform[3] = {153, 138, 138};
const uint8_t kInitCbfLuma[2] = {111, 141};
const uint8_t kInitCbfChroma[4] = {94, 138, 182, 154};
const uint8_t kInitLastPrefix[18] = {110, 110, 124, 125, 140, 153, 125, 127, 140,
                                     109, 111, 143, 127, 111, 79,  108, 123, 63};
const uint8_t kInitCsbf[4] = {91, 171, 134, 141};
const uint8_t kInitSig[42] = {111, 111, 125, 110, 110, 94,  124, 108, 124, 107, 125, 141, 179, 153,
                              125, 107, 125, 141, 179, 153, 125, 107, 125, 141, 179, 153, 125, 140,
                              139, 182, 182, 152, 136, 152, 136, 153, 136, 139, 111, 136, 139, 111};
const uint8_t kInitGreater1[24] = {140, 92,  137, 138, 140, 152, 138, 139, 153, 74,  149, 92,
                                   139, 107, 122, 152, 140, 179, 166, 182, 140, 227, 122, 197};
const uint8_t kInitGreater2[6] = {138, 153, 136, 167, 152, 152};

struct Contexts {
    Ctx sao_merge, sao_type, split_cu[3], part_mode, prev_intra_luma, intra_chroma, split_transform[3], cbf_luma[2],
        cbf_chroma[4], last_x[18], last_y[18], csbf[4], sig[42], greater1[24], greater2[6];
    void init(int qp) {
        sao_merge.init(kInitSaoMerge, qp);
        sao_type.init(kInitSaoType, qp);
        for (int i = 0; i < 3; i++) split_cu[i].init(kInitSplitCu[i], qp);
        part_mode.init(kInitPartMode, qp);
        prev_intra_luma.init(kInitPrevIntraLuma, qp);
        intra_chroma.init(kInitIntraChroma, qp);
        for (int i = 0; i < 3; i++) split_transform[i].init(kInitSplitTransform[i], qp);
        for (int i = 0; i < 2; i++) cbf_luma[i].init(kInitCbfLuma[i], qp);
        for (int i = 0; i < 4; i++) cbf_chroma[i].init(kInitCbfChroma[i], qp);
        for (int i = 0; i < 18; i++) {
            last_x[i].init(kInitLastPrefix[i], qp);
            last_y[i].init(kInitLastPrefix[i], qp);
        }
        for (int i = 0; i < 4; i++) csbf[i].init(kInitCsbf[i], qp);
        for (int i = 0; i < 42; i++) sig[i].init(kInitSig[i], qp);
        for (int i = 0; i < 24; i++) greater1[i].init(kInitGreater1[i], qp);
        for (int i = 0; i < 6; i++) greater2[i].init(kInitGreater2[i], qp);
    }
};

}  // namespace

namespace {

// ---- parameter sets (7.3.2) ---------------------------------------------------------------
void profile_tier_level(Bits& b) {
    b.put(0, 2);           // general_profile_space
    b.put(0, 1);           // general_tier_flag
    b.put(1, 5);           // general_profile_idc: Main
    for (int j = 0; j < 32; j++) b.bit(j == 1 || j == 2);   // compatible with Main and Main 10
    b.bit(1);              // general_progressive_source_flag
    b.bit(0);              // general_interlaced_source_flag
    b.bit(0);              // general_non_packed_constraint_flag
    b.bit(1);              // general_frame_only_constraint_flag
    b.put(0, 32);          // general_reserved_zero_43bits (and general_inbld_flag / reserved bit)
    b.put(0, 12);
    b.put(120, 8);         // general_level_idc: 4
}

struct Params {
    int W, H, log2_ctb, sao;
    int log2_max_tb() const { return std::min(5, log2_ctb); }
};

std::vector<uint8_t> vps() {
    Bits b;
    b.put(0, 4);           // vps_video_parameter_set_id
    b.bit(1);              // vps_base_layer_internal_flag
    b.bit(1);              // vps_base_layer_available_flag
    b.put(0, 6);           // vps_max_layers_minus1
    b.put(0, 3);           // vps_max_sub_layers_minus1
    b.bit(1);              // vps_temporal_id_nesting_flag
    b.put(0xFFFF, 16);     // vps_reserved_0xffff_16bits
    profile_tier_level(b);
    b.bit(1);              // vps_sub_layer_ordering_info_present_flag
    b.ue(1);               // vps_max_dec_pic_buffering_minus1
    b.ue(0);               // vps_max_num_reorder_pics
    b.ue(0);               // vps_max_latency_increase_plus1
    b.put(0, 6);           // vps_max_layer_id
    b.ue(0);               // vps_num_layer_sets_minus1
    b.bit(0);              // vps_timing_info_present_flag
    b.bit(0);              // vps_extension_flag
    b.trailing();
    return b.buf;
}

std::vector<uint8_t> sps(const Params& p) {
    Bits b;
    b.put(0, 4);           // sps_video_parameter_set_id
    b.put(0, 3);           // sps_max_sub_layers_minus1
    b.bit(1);              // sps_temporal_id_nesting_flag
    profile_tier_level(b);
    b.ue(0);               // sps_seq_parameter_set_id
    b.ue(1);               // chroma_format_idc: 4:2:0
    b.ue((uint32_t)p.W);   // pic_width_in_luma_samples
    b.ue((uint32_t)p.H);   // pic_height_in_luma_samples
    b.bit(0);              // conformance_window_flag
    b.ue(0);               // bit_depth_luma_minus8
    b.ue(0);               // bit_depth_chroma_minus8
    b.ue(4);               // log2_max_pic_order_cnt_lsb_minus4
    b.bit(1);              // sps_sub_layer_ordering_info_present_flag
    b.ue(1);               // sps_max_dec_pic_buffering_minus1
    b.ue(0);               // sps_max_num_reorder_pics
    b.ue(0);               // sps_max_latency_increase_plus1
    b.ue(0);               // log2_min_luma_coding_block_size_minus3: 8x8
    b.ue((uint32_t)(p.log2_ctb - 3));        // log2_diff_max_min_luma_coding_block_size
    b.ue(0);               // log2_min_luma_transform_block_size_minus2: 4x4
    b.ue((uint32_t)(p.log2_max_tb() - 2));   // log2_diff_max_min_luma_transform_block_size
    b.ue(1);               // max_transform_hierarchy_depth_inter
    b.ue(1);               // max_transform_hierarchy_depth_intra
    b.bit(0);              // scaling_list_enabled_flag
    b.bit(0);              // amp_enabled_flag
    b.bit(p.sao ? 1 : 0);  // sample_adaptive_offset_enabled_flag
    b.bit(0);              // pcm_enabled_flag
    b.ue(0);               // num_short_term_ref_pic_sets
    b.bit(0);              // long_term_ref_pics_present_flag
    b.bit(0);              // sps_temporal_mvp_enabled_flag
    b.bit(1);              // strong_intra_smoothing_enabled_flag
    b.bit(0);              // vui_parameters_present_flag
    b.bit(0);              // sps_extension_present_flag
    b.trailing();
    return b.buf;
}

std::vector<uint8_t> pps() {
    Bits b;
    b.ue(0);               // pps_pic_parameter_set_id
    b.ue(0);               // pps_seq_parameter_set_id
    b.bit(0);              // dependent_slice_segments_enabled_flag
    b.bit(0);              // output_flag_present_flag
    b.put(0, 3);           // num_extra_slice_header_bits
    b.bit(0);              // sign_data_hiding_enabled_flag
    b.bit(0);              // cabac_init_present_flag
    b.ue(0);               // num_ref_idx_l0_default_active_minus1
    b.ue(0);               // num_ref_idx_l1_default_active_minus1
    b.se(0);               // init_qp_minus26
    b.bit(0);              // constrained_intra_pred_flag
    b.bit(0);              // transform_skip_enabled_flag
    b.bit(0);              // cu_qp_delta_enabled_flag
    b.se(0);               // pps_cb_qp_offset
    b.se(0);               // pps_cr_qp_offset
    b.bit(0);              // pps_slice_chroma_qp_offsets_present_flag
    b.bit(0);              // weighted_pred_flag
    b.bit(0);              // weighted_bipred_flag
    b.bit(0);              // transquant_bypass_enabled_flag
    b.bit(0);              // tiles_enabled_flag
    b.bit(0);              // entropy_coding_sync_enabled_flag
    b.bit(1);              // pps_loop_filter_across_slices_enabled_flag
    b.bit(0);              // deblocking_filter_control_present_flag
    b.bit(0);              // pps_scaling_list_data_present_flag
    b.bit(0);              // lists_modification_present_flag
    b.ue(0);               // log2_parallel_merge_level_minus2
    b.bit(0);              // slice_segment_header_extension_present_flag
    b.bit(0);              // pps_extension_present_flag
    b.trailing();
    return b.buf;
}

// chroma QP of 4:2:0 (8.6.1, table 8-10) for the records
int chroma_qp(int qpi) {
    static const int tab[14] = {29, 30, 31, 32, 33, 33, 34, 34, 35, 35, 36, 36, 37, 37};
    qpi = std::min(57, std::max(0, qpi));
    return qpi < 30 ? qpi : (qpi > 43 ? qpi - 6 : tab[qpi - 30]);
}

}  // namespace

namespace {

// ---- one picture ----------------------------------------------------------------------------
struct Picture {
    const hevcgen_cfg_t& cfg;
    std::mt19937_64& rng;
    Params p;
    int qp = 26;
    int wctb = 0, hctb = 0;
    std::vector<uint8_t> depth8;   // CtDepth per 8x8 unit
    std::vector<uint8_t> mode4;    // IntraPredModeY per 4x4 luma unit
    Contexts C;
    Cabac E;
    std::vector<hevc_tu_t> tus;
    std::vector<int16_t> coeffs;

    Picture(const hevcgen_cfg_t& c, std::mt19937_64& r, const Params& pp) : cfg(c), rng(r), p(pp) {}

    double u01() { return std::uniform_real_distribution<double>(0.0, 1.0)(rng); }
    int uni(int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); }

    // split_cu_flag context: neighbours deeper than this node (9.3.4.2.2)
    void coding_quadtree(int x0, int y0, int log2, int depth) {
        const int size = 1 << log2;
        bool split;
        if (x0 + size <= p.W && y0 + size <= p.H && log2 > 3) {
            split = u01() < cfg.p_split;
            const int w8 = p.W / 8;
            const int inc = (x0 > 0 && depth8[(size_t)(y0 / 8) * w8 + (x0 - 1) / 8] > depth) +
                            (y0 > 0 && depth8[(size_t)((y0 - 1) / 8) * w8 + x0 / 8] > depth);
            E.decision(C.split_cu[inc], split);
        } else {
            split = log2 > 3;
        }
        if (split) {
            const int h = size / 2;
            for (int k = 0; k < 4; k++) {
                const int x = x0 + (k & 1) * h, y = y0 + (k >> 1) * h;
                if (x < p.W && y < p.H) coding_quadtree(x, y, log2 - 1, depth + 1);
            }
            return;
        }
        const int w8 = p.W / 8;
        for (int y = y0 / 8; y < (y0 + size) / 8; y++)
            for (int x = x0 / 8; x < (x0 + size) / 8; x++) depth8[(size_t)y * w8 + x] = (uint8_t)depth;
        coding_unit(x0, y0, log2);
    }

    // candModeList of a prediction block (8.4.2)
    void mpm(int xPb, int yPb, int cand[3]) {
        const int w4 = p.W / 4;
        const int a = xPb > 0 ? mode4[(size_t)(yPb / 4) * w4 + (xPb - 1) / 4] : 1;
        const bool above_in_ctb_row = yPb - 1 >= ((yPb >> p.log2_ctb) << p.log2_ctb);
        const int b = (yPb > 0 && above_in_ctb_row) ? mode4[(size_t)((yPb - 1) / 4) * w4 + xPb / 4] : 1;
        if (a == b) {
            if (a < 2) {
                cand[0] = 0;
                cand[1] = 1;
                cand[2] = 26;
            } else {
                cand[0] = a;
                cand[1] = 2 + ((a + 29) % 32);
                cand[2] = 2 + ((a - 2 + 1) % 32);
            }
        } else {
            cand[0] = a;
            cand[1] = b;
            cand[2] = (a != 0 && b != 0) ? 0 : ((a != 1 && b != 1) ? 1 : 26);
        }
    }

    void coding_unit(int x0, int y0, int log2) {
        const int size = 1 << log2;
        const bool nxn = log2 == 3 && u01() < cfg.p_nxn;
        if (log2 == 3) E.decision(C.part_mode, nxn ? 0 : 1);   // part_mode: PART_2Nx2N = 1, PART_NxN = 0
        const int npb = nxn ? 4 : 1, pbs = nxn ? size / 2 : size;
        int mode[4], flag[4], idx[4];
        const int w4 = p.W / 4;
        for (int k = 0; k < npb; k++) {
            const int xp = x0 + (k & 1) * pbs, yp = y0 + (k >> 1) * pbs;
            mode[k] = uni(0, 34);
            int cand[3];
            mpm(xp, yp, cand);
            flag[k] = 0;
            for (int q = 0; q < 3; q++)
                if (cand[q] == mode[k]) {
                    flag[k] = 1;
                    idx[k] = q;
                }
            if (!flag[k]) {
                std::sort(cand, cand + 3);
                int rem = mode[k];
                for (int q = 2; q >= 0; q--)
                    if (mode[k] > cand[q]) rem--;
                idx[k] = rem;
            }
            for (int y = yp / 4; y < (yp + pbs) / 4; y++)
                for (int x = xp / 4; x < (xp + pbs) / 4; x++) mode4[(size_t)y * w4 + x] = (uint8_t)mode[k];
        }
        for (int k = 0; k < npb; k++) E.decision(C.prev_intra_luma, flag[k]);
        for (int k = 0; k < npb; k++) {
            if (flag[k]) {   // mpm_idx: truncated rice, cMax 2, bypass
                E.bypass(idx[k] > 0);
                if (idx[k] > 0) E.bypass(idx[k] > 1);
            } else {
                E.bypass_bits((uint32_t)idx[k], 5);   // rem_intra_luma_pred_mode
            }
        }
        const int chroma_syntax = uni(0, 4);
        E.decision(C.intra_chroma, chroma_syntax == 4 ? 0 : 1);
        if (chroma_syntax != 4) E.bypass_bits((uint32_t)chroma_syntax, 2);
        int cmode = mode[0];
        if (chroma_syntax != 4) {
            static const int cand[4] = {0, 26, 10, 1};
            cmode = cand[chroma_syntax] == mode[0] ? 34 : cand[chroma_syntax];
        }
        const int max_depth = 1 + (nxn ? 1 : 0);   // max_transform_hierarchy_depth_intra + IntraSplitFlag
        transform_tree(x0, y0, x0, y0, log2, 0, 0, nxn, max_depth, cmode, true, true);
    }

    void record(int c, int x, int y, int log2, int mode, bool coded) {
        hevc_tu_t t{};
        t.x = (uint16_t)x;
        t.y = (uint16_t)y;
        t.log2_size = (uint8_t)log2;
        t.c_idx = (uint8_t)c;
        t.qp = (uint8_t)(c ? chroma_qp(qp) : qp);
        t.flags = (uint8_t)(HEVC_TU_INTRA | (coded ? HEVC_TU_CODED : 0));
        t.intra_mode = (uint8_t)mode;
        t.coeff_offset = 0;
        if (coded) {
            t.coeff_offset = (uint32_t)coeffs.size();
            coeffs.resize(coeffs.size() + ((size_t)1 << (2 * log2)), 0);
        }
        tus.push_back(t);
    }

    void transform_tree(int x0, int y0, int xb, int yb, int log2, int depth, int blk, bool nxn, int max_depth,
                        int cmode, bool parent_cb, bool parent_cr) {
        bool split;
        if (log2 <= p.log2_max_tb() && log2 > 2 && depth < max_depth && !(nxn && depth == 0)) {
            split = u01() < cfg.p_tu_split;
            E.decision(C.split_transform[5 - log2], split);
        } else {
            split = log2 > p.log2_max_tb() || (nxn && depth == 0);
        }
        bool cb = false, cr = false;
        if (log2 > 2) {
            if (depth == 0 || parent_cb) {
                cb = u01() < cfg.p_cbf;
                E.decision(C.cbf_chroma[depth], cb);
            }
            if (depth == 0 || parent_cr) {
                cr = u01() < cfg.p_cbf;
                E.decision(C.cbf_chroma[depth], cr);
            }
        } else {
            cb = parent_cb;
            cr = parent_cr;
        }
        if (split) {
            const int h = 1 << (log2 - 1);
            for (int k = 0; k < 4; k++)
                transform_tree(x0 + (k & 1) * h, y0 + (k >> 1) * h, x0, y0, log2 - 1, depth + 1, k, nxn, max_depth, cmode,
                               cb, cr);
            return;
        }
        const bool cbf_luma = u01() < cfg.p_cbf;
        E.decision(C.cbf_luma[depth == 0 ? 1 : 0], cbf_luma);
        const int w4 = p.W / 4;
        record(0, x0, y0, log2, mode4[(size_t)(y0 / 4) * w4 + x0 / 4], cbf_luma);
        if (cbf_luma) residual(x0, y0, log2, 0, mode4[(size_t)(y0 / 4) * w4 + x0 / 4]);
        if (log2 > 2) {
            for (int c = 1; c <= 2; c++) {
                const bool f = c == 1 ? cb : cr;
                record(c, x0 / 2, y0 / 2, log2 - 1, cmode, f);
                if (f) residual(x0 / 2, y0 / 2, log2 - 1, c, cmode);
            }
        } else if (blk == 3) {
            for (int c = 1; c <= 2; c++) {
                const bool f = c == 1 ? cb : cr;
                record(c, xb / 2, yb / 2, 2, cmode, f);
                if (f) residual(xb / 2, yb / 2, 2, c, cmode);
            }
        }
    }

    void residual(int x0, int y0, int log2, int c, int mode);   // below

    std::vector<uint8_t> slice_data_and_header(int idr) {
        (void)idr;
        Bits b;
        b.bit(1);            // first_slice_segment_in_pic_flag
        b.bit(0);            // no_output_of_prior_pics_flag
        b.ue(0);             // slice_pic_parameter_set_id
        b.ue(2);             // slice_type: I
        if (p.sao) {
            b.bit(1);        // slice_sao_luma_flag
            b.bit(1);        // slice_sao_chroma_flag
        }
        b.se(qp - 26);       // slice_qp_delta
        b.bit(1);            // slice_loop_filter_across_slices_enabled_flag
        b.trailing();        // byte_alignment()
        C.init(qp);
        E.start(&b);
        const int nctb = wctb * hctb;
        for (int a = 0; a < nctb; a++) {
            const int rx = a % wctb, ry = a / wctb;
            if (p.sao) sao(rx, ry);
            coding_quadtree(rx << p.log2_ctb, ry << p.log2_ctb, p.log2_ctb, 0);
            E.terminate(a == nctb - 1);   // end_of_slice_segment_flag
        }
        b.align_zero();
        return b.buf;
    }

    void sao(int rx, int ry);   // below
};

}  // namespace

namespace {

// scan orders (6.5.3-6.5.5): ScanOrder[log2 size][scanIdx][pos] = (x, y)
struct Scans {
    std::vector<std::pair<int, int>> s[4][3];   // log2 size 0..3 (1x1 .. 8x8), diag / hor / ver
    Scans() {
        for (int l = 0; l < 4; l++) {
            const int n = 1 << l;
            auto& d = s[l][0];
            int x = 0, y = 0;
            while ((int)d.size() < n * n) {
                while (y >= 0) {
                    if (x < n && y < n) d.push_back({x, y});
                    y--;
                    x++;
                }
                y = x;
                x = 0;
            }
            for (int yy = 0; yy < n; yy++)
                for (int xx = 0; xx < n; xx++) s[l][1].push_back({xx, yy});
            for (int xx = 0; xx < n; xx++)
                for (int yy = 0; yy < n; yy++) s[l][2].push_back({xx, yy});
        }
    }
};
const Scans& scans() {
    static const Scans sc;
    return sc;
}

const int kGroupIdx[32] = {0, 1, 2, 3, 4, 4, 5, 5, 6, 6, 6, 6, 7, 7, 7, 7,
                           8, 8, 8, 8, 8, 8, 8, 8, 9, 9, 9, 9, 9, 9, 9, 9};
const int kMinInGroup[10] = {0, 1, 2, 3, 4, 6, 8, 12, 16, 24};
const int kCtxIdxMap4x4[16] = {0, 1, 4, 5, 2, 3, 4, 5, 6, 6, 8, 8, 7, 7, 8, 8};

}  // namespace

// residual_coding() (7.3.8.11) of one transform block: levels drawn and CABAC-coded.
void Picture::residual(int x0, int y0, int log2, int c, int mode) {
    const int n = 1 << log2, ls = log2 - 2, nsb = 1 << ls;
    int scan_idx = 0;
    if (log2 == 2 || (log2 == 3 && c == 0)) scan_idx = (mode >= 6 && mode <= 14) ? 2 : ((mode >= 22 && mode <= 30) ? 1 : 0);
    const auto& sb_scan = scans().s[ls][scan_idx];
    const auto& pos_scan = scans().s[2][scan_idx];
    auto at = [&](int i) {   // scan index -> (x, y) in the block
        const auto sb = sb_scan[(size_t)(i >> 4)];
        const auto ps = pos_scan[(size_t)(i & 15)];
        return std::make_pair((sb.first << 2) + ps.first, (sb.second << 2) + ps.second);
    };
    // draw: the last significant position, and levels before it
    int16_t* lv = coeffs.data() + tus.back().coeff_offset;
    const int total = n * n;
    int last = std::min(total - 1, (int)(std::pow(u01(), 2.0) * total));
    auto draw_level = [&]() {
        int a = 1;
        while (a < cfg.max_level && u01() < 0.45) a += 1 + (u01() < 0.2 ? uni(0, 20) : 0);
        a = std::min(a, cfg.max_level);
        return (int16_t)(u01() < 0.5 ? -a : a);
    };
    for (int i = 0; i <= last; i++) {
        const auto xy = at(i);
        if (i == last || u01() < cfg.p_sig) lv[xy.second * n + xy.first] = draw_level();
    }
    // last_sig_coeff_x/y (swapped for the vertical scan) and their contexts (9.3.4.2.3)
    const auto lxy = at(last);
    const int lx = scan_idx == 2 ? lxy.second : lxy.first, ly = scan_idx == 2 ? lxy.first : lxy.second;
    const int off = c ? 15 : 3 * (log2 - 2) + ((log2 - 1) >> 2), shift = c ? log2 - 2 : (log2 + 1) >> 2;
    const int cmax = (log2 << 1) - 1;
    const int px = kGroupIdx[lx], py = kGroupIdx[ly];
    for (int k = 0; k < std::min(px + 1, cmax); k++) E.decision(C.last_x[off + (k >> shift)], k < px);
    for (int k = 0; k < std::min(py + 1, cmax); k++) E.decision(C.last_y[off + (k >> shift)], k < py);
    if (px > 3) E.bypass_bits((uint32_t)(lx - kMinInGroup[px]), (px >> 1) - 1);
    if (py > 3) E.bypass_bits((uint32_t)(ly - kMinInGroup[py]), (py >> 1) - 1);
    // coded sub-block flags as the decoder sees them: 1 for the last and the first sub-block
    std::vector<uint8_t> csbf((size_t)nsb * nsb, 0);
    const int last_sb = last >> 4;
    for (int i = 0; i <= last; i++) {
        const auto xy = at(i);
        if (lv[xy.second * n + xy.first]) csbf[(size_t)(xy.second >> 2) * nsb + (xy.first >> 2)] = 1;
    }
    {
        const auto sb = sb_scan[(size_t)last_sb];
        csbf[(size_t)sb.second * nsb + sb.first] = 1;
    }
    int c1 = 1;
    for (int i = last_sb; i >= 0; i--) {
        const int xs = sb_scan[(size_t)i].first, ys = sb_scan[(size_t)i].second;
        const int right = xs + 1 < nsb ? csbf[(size_t)ys * nsb + xs + 1] : 0;
        const int below = ys + 1 < nsb ? csbf[(size_t)(ys + 1) * nsb + xs] : 0;
        bool infer_dc = false;
        if (i < last_sb && i > 0) {
            E.decision(C.csbf[std::min(right + below, 1) + (c ? 2 : 0)], csbf[(size_t)ys * nsb + xs]);
            infer_dc = true;
        }
        const bool coded = i == last_sb || i == 0 || csbf[(size_t)ys * nsb + xs];
        std::vector<int> sig;   // levels of the significant positions, in coding order
        if (i == last_sb) sig.push_back(lv[lxy.second * n + lxy.first]);
        const int prev_csbf = right + 2 * below;
        for (int q = (i == last_sb) ? (last & 15) - 1 : 15; q >= 0 && coded; q--) {
            const int xc = (xs << 2) + pos_scan[(size_t)q].first, yc = (ys << 2) + pos_scan[(size_t)q].second;
            const int v = lv[yc * n + xc];
            if (q > 0 || !infer_dc) {
                int sctx;   // sig_coeff_flag context (9.3.4.2.5)
                if (log2 == 2) sctx = kCtxIdxMap4x4[(yc << 2) + xc];
                else if (xc + yc == 0) sctx = 0;
                else {
                    const int xp = xc & 3, yp = yc & 3;
                    if (prev_csbf == 0) sctx = (xp + yp == 0) ? 2 : (xp + yp < 3) ? 1 : 0;
                    else if (prev_csbf == 1) sctx = yp == 0 ? 2 : (yp == 1 ? 1 : 0);
                    else if (prev_csbf == 2) sctx = xp == 0 ? 2 : (xp == 1 ? 1 : 0);
                    else sctx = 2;
                    if (c == 0) {
                        if (xs + ys > 0) sctx += 3;
                        sctx += log2 == 3 ? (scan_idx == 0 ? 9 : 15) : 21;
                    } else {
                        sctx += log2 == 3 ? 9 : 12;
                    }
                }
                E.decision(C.sig[c ? 27 + sctx : sctx], v != 0);
                if (v) infer_dc = false;
            }
            if (v) sig.push_back(v);
        }
        if (sig.empty()) continue;
        // greater-1 / greater-2 flags (9.3.4.2.6, 9.3.4.2.7), signs, remainders (9.3.3.11)
        int ctx_set = (i > 0 && c == 0) ? 2 : 0;
        if (c1 == 0) ctx_set++;
        c1 = 1;
        const int ns = (int)sig.size(), n1 = std::min(ns, 8);
        int first_c2 = -1;
        for (int k = 0; k < n1; k++) {
            const int g1 = std::abs(sig[(size_t)k]) > 1;
            E.decision(C.greater1[(c ? 16 : 0) + ctx_set * 4 + c1], g1);
            if (g1) {
                c1 = 0;
                if (first_c2 < 0) first_c2 = k;
            } else if (c1 > 0 && c1 < 3) {
                c1++;
            }
        }
        if (first_c2 >= 0) E.decision(C.greater2[(c ? 4 : 0) + ctx_set], std::abs(sig[(size_t)first_c2]) > 2);
        for (int k = 0; k < ns; k++) E.bypass(sig[(size_t)k] < 0);
        int rice = 0;
        for (int k = 0; k < ns; k++) {
            const int a = std::abs(sig[(size_t)k]);
            const int base = k < 8 ? 2 + (k == first_c2 ? 1 : 0) : 1;
            if (a < base) continue;
            uint32_t v = (uint32_t)(a - base);
            if (v < (3u << rice)) {
                const uint32_t q = v >> rice;
                for (uint32_t b = 0; b < q; b++) E.bypass(1);
                E.bypass(0);
                E.bypass_bits(v & ((1u << rice) - 1u), rice);
            } else {
                int len = rice;
                v -= 3u << rice;
                while (v >= (1u << len)) {
                    v -= 1u << len;
                    len++;
                }
                for (int b = 0; b < 3 + len - rice; b++) E.bypass(1);
                E.bypass(0);
                E.bypass_bits(v, len);
            }
            if (a > 3 * (1 << rice)) rice = std::min(rice + 1, 4);
        }
    }
}

// sao() (7.3.8.3) of one CTB: merges, types, offsets, band positions, edge classes.
void Picture::sao(int rx, int ry) {
    bool merge = false;
    if (rx > 0) {
        merge = u01() < 0.3;
        E.decision(C.sao_merge, merge);
    }
    if (!merge && ry > 0) {
        merge = u01() < 0.3;
        E.decision(C.sao_merge, merge);
    }
    if (merge) return;
    int type = 0;
    for (int c = 0; c < 3; c++) {
        if (c < 2) {   // sao_type_idx: TR cMax 2, first bin context-coded
            type = uni(0, 2);
            E.decision(C.sao_type, type != 0);
            if (type) E.bypass(type == 2);
        }
        if (!type) continue;
        int abs_v[4];
        for (int k = 0; k < 4; k++) {   // sao_offset_abs: TR cMax 7, bypass
            abs_v[k] = uni(0, 7);
            for (int b = 0; b < abs_v[k]; b++) E.bypass(1);
            if (abs_v[k] < 7) E.bypass(0);
        }
        if (type == 1) {
            for (int k = 0; k < 4; k++)
                if (abs_v[k]) E.bypass(uni(0, 1));
            E.bypass_bits((uint32_t)uni(0, 31), 5);   // sao_band_position
        } else if (c < 2) {
            E.bypass_bits((uint32_t)uni(0, 3), 2);    // sao_eo_class
        }
    }
}

extern "C" {

void hevcgen_default_cfg(hevcgen_cfg_t* cfg, int32_t width, int32_t height, uint64_t seed) {
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->width = width;
    cfg->height = height;
    cfg->seed = seed;
    cfg->pictures = 2;
    cfg->log2_ctb = 6;
    cfg->p_split = 0.6;
    cfg->p_nxn = 0.3;
    cfg->p_tu_split = 0.3;
    cfg->p_cbf = 0.5;
    cfg->p_sig = 0.3;
    cfg->max_level = 200;
    cfg->qp_min = 22;
    cfg->qp_max = 40;
    cfg->sao = 1;
}

hevcgen_stream_t* hevcgen_stream(const hevcgen_cfg_t* cfg) {
    if (!cfg || cfg->width <= 0 || cfg->height <= 0 || (cfg->width & 7) || (cfg->height & 7) || cfg->pictures < 1 ||
        cfg->log2_ctb < 4 || cfg->log2_ctb > 6 || cfg->max_level < 1 || cfg->qp_min < 0 || cfg->qp_max > 51 ||
        cfg->qp_min > cfg->qp_max)
        return nullptr;
    std::mt19937_64 rng(cfg->seed);
    Params p{cfg->width, cfg->height, cfg->log2_ctb, cfg->sao ? 1 : 0};
    std::vector<uint8_t> out;
    nal(out, 32, vps());
    nal(out, 33, sps(p));
    nal(out, 34, pps());
    auto* s = static_cast<hevcgen_stream_t*>(std::calloc(1, sizeof(hevcgen_stream_t)));
    s->pictures = cfg->pictures;
    s->num_tus = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->tus = static_cast<hevc_tu_t**>(std::calloc((size_t)cfg->pictures, sizeof(hevc_tu_t*)));
    s->num_coeffs = static_cast<uint64_t*>(std::calloc((size_t)cfg->pictures, sizeof(uint64_t)));
    s->coeffs = static_cast<int16_t**>(std::calloc((size_t)cfg->pictures, sizeof(int16_t*)));
    for (int k = 0; k < cfg->pictures; k++) {
        Picture pic(*cfg, rng, p);
        pic.qp = std::uniform_int_distribution<int>(cfg->qp_min, cfg->qp_max)(rng);
        pic.wctb = (p.W + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
        pic.hctb = (p.H + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
        pic.depth8.assign((size_t)(p.W / 8) * (p.H / 8), 0);
        pic.mode4.assign((size_t)(p.W / 4) * (p.H / 4), 1);
        pic.coeffs.reserve((size_t)p.W * p.H * 3 / 2);
        nal(out, 19, pic.slice_data_and_header(k));   // IDR_W_RADL
        s->num_tus[k] = (int32_t)pic.tus.size();
        s->tus[k] = static_cast<hevc_tu_t*>(std::malloc(sizeof(hevc_tu_t) * std::max<size_t>(1, pic.tus.size())));
        std::memcpy(s->tus[k], pic.tus.data(), sizeof(hevc_tu_t) * pic.tus.size());
        s->num_coeffs[k] = pic.coeffs.size();
        s->coeffs[k] = static_cast<int16_t*>(std::malloc(sizeof(int16_t) * std::max<size_t>(1, pic.coeffs.size())));
        std::memcpy(s->coeffs[k], pic.coeffs.data(), sizeof(int16_t) * pic.coeffs.size());
    }
    s->size = out.size();
    s->bytes = static_cast<uint8_t*>(std::malloc(out.size()));
    std::memcpy(s->bytes, out.data(), out.size());
    return s;
}

void hevcgen_stream_free(hevcgen_stream_t* s) {
    if (!s) return;
    for (int k = 0; k < s->pictures; k++) {
        std::free(s->tus[k]);
        std::free(s->coeffs[k]);
    }
    std::free(s->num_tus);
    std::free(s->tus);
    std::free(s->num_coeffs);
    std::free(s->coeffs);
    std::free(s->bytes);
    std::free(s);
}

}  // extern "C"
