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

// Context initialisation values, 9.3.2.2 tables 9-5 .. 9-37, per initType: [0] I slices,
// [1] P slices (B slices with cabac_init_flag), [2] B slices (P slices with cabac_init_flag).
// The syntax elements of inter CUs have no initType-0 values (0 there: never used).
const uint8_t kInitSaoMerge[3] = {153, 153, 153};
const uint8_t kInitSaoType[3] = {200, 185, 160};
const uint8_t kInitSplitCu[3][3] = {{139, 141, 157}, {107, 139, 126}, {107, 139, 126}};
const uint8_t kInitSkip[3][3] = {{0, 0, 0}, {197, 185, 201}, {197, 185, 201}};
const uint8_t kInitPredMode[3] = {0, 149, 134};
const uint8_t kInitPartMode[3][4] = {{184, 0, 0, 0}, {154, 139, 154, 154}, {154, 139, 154, 154}};
const uint8_t kInitPrevIntraLuma[3] = {184, 154, 183};
const uint8_t kInitIntraChroma[3] = {63, 152, 152};
const uint8_t kInitRqtRootCbf[3] = {0, 79, 79};
const uint8_t kInitMergeFlag[3] = {0, 110, 154};
const uint8_t kInitMergeIdx[3] = {0, 122, 137};
const uint8_t kInitInterPredIdc[5] = {95, 79, 63, 31, 31};   // initType 1 and 2
const uint8_t kInitRefIdx[2] = {153, 153};                   // initType 1 and 2
const uint8_t kInitMvpFlag = 168;                            // initType 1 and 2
const uint8_t kInitMvdGreater0[3] = {0, 140, 169};
const uint8_t kInitMvdGreater1[3] = {0, 198, 198};
const uint8_t kInitSplitTransform[3][3] = {{153, 138, 138}, {124, 138, 94}, {224, 167, 122}};
const uint8_t kInitCbfLuma[3][2] = {{111, 141}, {153, 111}, {153, 111}};
const uint8_t kInitCbfChroma[3][4] = {{94, 138, 182, 154}, {149, 107, 167, 154}, {149, 92, 167, 154}};
const uint8_t kInitLastPrefix[3][18] = {
    {110, 110, 124, 125, 140, 153, 125, 127, 140, 109, 111, 143, 127, 111, 79, 108, 123, 63},
    {125, 110, 94, 110, 95, 79, 125, 111, 110, 78, 110, 111, 111, 95, 94, 108, 123, 108},
    {125, 110, 124, 110, 95, 94, 125, 111, 111, 79, 125, 126, 111, 111, 79, 108, 123, 93}};
const uint8_t kInitCsbf[3][4] = {{91, 171, 134, 141}, {121, 140, 61, 154}, {121, 140, 61, 154}};
const uint8_t kInitSig[3][42] = {
    {111, 111, 125, 110, 110, 94,  124, 108, 124, 107, 125, 141, 179, 153, 125, 107, 125, 141, 179, 153, 125,
     107, 125, 141, 179, 153, 125, 140, 139, 182, 182, 152, 136, 152, 136, 153, 136, 139, 111, 136, 139, 111},
    {155, 154, 139, 153, 139, 123, 123, 63,  153, 166, 183, 140, 136, 153, 154, 166, 183, 140, 136, 153, 154,
     166, 183, 140, 136, 153, 154, 170, 153, 123, 123, 107, 121, 107, 121, 167, 151, 183, 140, 151, 183, 140},
    {170, 154, 139, 153, 139, 123, 123, 63,  124, 166, 183, 140, 136, 153, 154, 166, 183, 140, 136, 153, 154,
     166, 183, 140, 136, 153, 154, 170, 153, 138, 138, 122, 121, 122, 121, 167, 151, 183, 140, 151, 183, 140}};
const uint8_t kInitGreater1[3][24] = {
    {140, 92, 137, 138, 140, 152, 138, 139, 153, 74, 149, 92, 139, 107, 122, 152, 140, 179, 166, 182, 140, 227, 122, 197},
    {154, 196, 196, 167, 154, 152, 167, 182, 182, 134, 149, 136, 153, 121, 136, 137, 169, 194, 166, 167, 154, 167, 137, 182},
    {154, 196, 167, 167, 154, 152, 167, 182, 182, 134, 149, 136, 153, 121, 136, 122, 169, 208, 166, 167, 154, 152, 167, 182}};
const uint8_t kInitGreater2[3][6] = {{138, 153, 136, 167, 152, 152}, {107, 167, 91, 122, 107, 167}, {107, 167, 91, 107, 107, 167}};

struct Contexts {
    Ctx sao_merge, sao_type, split_cu[3], skip[3], pred_mode, part_mode[4], prev_intra_luma, intra_chroma, rqt_root_cbf,
        merge_flag, merge_idx, inter_pred_idc[5], ref_idx[2], mvp_flag, mvd_greater0, mvd_greater1, split_transform[3],
        cbf_luma[2], cbf_chroma[4], last_x[18], last_y[18], csbf[4], sig[42], greater1[24], greater2[6];
    void init(int t, int qp) {   // t: initType
        sao_merge.init(kInitSaoMerge[t], qp);
        sao_type.init(kInitSaoType[t], qp);
        for (int i = 0; i < 3; i++) split_cu[i].init(kInitSplitCu[t][i], qp);
        for (int i = 0; i < 3; i++) skip[i].init(kInitSkip[t][i], qp);
        pred_mode.init(kInitPredMode[t], qp);
        for (int i = 0; i < 4; i++) part_mode[i].init(kInitPartMode[t][i], qp);
        prev_intra_luma.init(kInitPrevIntraLuma[t], qp);
        intra_chroma.init(kInitIntraChroma[t], qp);
        rqt_root_cbf.init(kInitRqtRootCbf[t], qp);
        merge_flag.init(kInitMergeFlag[t], qp);
        merge_idx.init(kInitMergeIdx[t], qp);
        for (int i = 0; i < 5; i++) inter_pred_idc[i].init(kInitInterPredIdc[i], qp);
        for (int i = 0; i < 2; i++) ref_idx[i].init(kInitRefIdx[i], qp);
        mvp_flag.init(kInitMvpFlag, qp);
        mvd_greater0.init(kInitMvdGreater0[t], qp);
        mvd_greater1.init(kInitMvdGreater1[t], qp);
        for (int i = 0; i < 3; i++) split_transform[i].init(kInitSplitTransform[t][i], qp);
        for (int i = 0; i < 2; i++) cbf_luma[i].init(kInitCbfLuma[t][i], qp);
        for (int i = 0; i < 4; i++) cbf_chroma[i].init(kInitCbfChroma[t][i], qp);
        for (int i = 0; i < 18; i++) {
            last_x[i].init(kInitLastPrefix[t][i], qp);
            last_y[i].init(kInitLastPrefix[t][i], qp);
        }
        for (int i = 0; i < 4; i++) csbf[i].init(kInitCsbf[t][i], qp);
        for (int i = 0; i < 42; i++) sig[i].init(kInitSig[t][i], qp);
        for (int i = 0; i < 24; i++) greater1[i].init(kInitGreater1[t][i], qp);
        for (int i = 0; i < 6; i++) greater2[i].init(kInitGreater2[t][i], qp);
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
    int inter = 0, dpb_minus1 = 1, amp = 0, tmvp = 0, wp = 0, depth_inter = 1;
    int log2_max_tb() const { return std::min(5, log2_ctb); }
};

std::vector<uint8_t> vps(const Params& p) {
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
    b.ue((uint32_t)p.dpb_minus1);            // vps_max_dec_pic_buffering_minus1
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
    b.ue((uint32_t)p.dpb_minus1);            // sps_max_dec_pic_buffering_minus1
    b.ue(0);               // sps_max_num_reorder_pics
    b.ue(0);               // sps_max_latency_increase_plus1
    b.ue(0);               // log2_min_luma_coding_block_size_minus3: 8x8
    b.ue((uint32_t)(p.log2_ctb - 3));        // log2_diff_max_min_luma_coding_block_size
    b.ue(0);               // log2_min_luma_transform_block_size_minus2: 4x4
    b.ue((uint32_t)(p.log2_max_tb() - 2));   // log2_diff_max_min_luma_transform_block_size
    b.ue((uint32_t)p.depth_inter);           // max_transform_hierarchy_depth_inter
    b.ue(1);               // max_transform_hierarchy_depth_intra
    b.bit(0);              // scaling_list_enabled_flag
    b.bit(p.amp ? 1 : 0);  // amp_enabled_flag
    b.bit(p.sao ? 1 : 0);  // sample_adaptive_offset_enabled_flag
    b.bit(0);              // pcm_enabled_flag
    b.ue(0);               // num_short_term_ref_pic_sets
    b.bit(0);              // long_term_ref_pics_present_flag
    b.bit(p.tmvp ? 1 : 0); // sps_temporal_mvp_enabled_flag
    b.bit(1);              // strong_intra_smoothing_enabled_flag
    b.bit(0);              // vui_parameters_present_flag
    b.bit(0);              // sps_extension_present_flag
    b.trailing();
    return b.buf;
}

std::vector<uint8_t> pps(const Params& p) {
    Bits b;
    b.ue(0);               // pps_pic_parameter_set_id
    b.ue(0);               // pps_seq_parameter_set_id
    b.bit(0);              // dependent_slice_segments_enabled_flag
    b.bit(0);              // output_flag_present_flag
    b.put(0, 3);           // num_extra_slice_header_bits
    b.bit(0);              // sign_data_hiding_enabled_flag
    b.bit(p.inter ? 1 : 0);   // cabac_init_present_flag (cabac_init_flag drawn per slice)
    b.ue(0);               // num_ref_idx_l0_default_active_minus1
    b.ue(0);               // num_ref_idx_l1_default_active_minus1
    b.se(0);               // init_qp_minus26
    b.bit(0);              // constrained_intra_pred_flag
    b.bit(0);              // transform_skip_enabled_flag
    b.bit(0);              // cu_qp_delta_enabled_flag
    b.se(0);               // pps_cb_qp_offset
    b.se(0);               // pps_cr_qp_offset
    b.bit(0);              // pps_slice_chroma_qp_offsets_present_flag
    b.bit(p.wp ? 1 : 0);   // weighted_pred_flag
    b.bit(p.wp ? 1 : 0);   // weighted_bipred_flag
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
// The reference picture state carried from one picture to the next.
struct GopState {
    std::vector<int> refs;   // POCs the next picture's RPS keeps, most recent first
    int tmvp_barrier = 0;    // POC of the last picture with slice_temporal_mvp_enabled_flag 0
};

struct Picture {
    const hevcgen_cfg_t& cfg;
    std::mt19937_64& rng;
    Params p;
    int qp = 26;
    int wctb = 0, hctb = 0;
    // the slice: type (0 B, 1 P, 2 I), active reference list sizes, MaxNumMergeCand
    int slice_type = 2, num_ref[2] = {0, 0}, max_merge = 5;
    bool mvd_l1_zero = false;
    std::vector<uint8_t> depth8;   // CtDepth per 8x8 unit
    std::vector<uint8_t> skip8;    // cu_skip_flag per 8x8 unit
    std::vector<uint8_t> mode4;    // IntraPredModeY per 4x4 luma unit (DC for inter CUs)
    Contexts C;
    Cabac E;
    std::vector<hevc_tu_t> tus;
    std::vector<int16_t> coeffs;
    std::vector<hevc_pu_t> pus;

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
        coding_unit(x0, y0, log2, depth);
    }

    // fill a per-unit map over a rectangle of luma samples
    static void fill(std::vector<uint8_t>& m, int unit, int stride, int x0, int y0, int w, int h, uint8_t v) {
        for (int y = y0 / unit; y < (y0 + h) / unit; y++)
            for (int x = x0 / unit; x < (x0 + w) / unit; x++) m[(size_t)y * stride + x] = v;
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

    // coding_unit() (7.3.8.5).  In a P/B slice: cu_skip_flag (context from the left and
    // above CUs' flags, 9.3.4.2.2), then pred_mode_flag; inter CUs go to inter_cu.
    void coding_unit(int x0, int y0, int log2, int depth) {
        const int size = 1 << log2;
        if (slice_type != 2) {
            const int w8 = p.W / 8;
            const bool skip = u01() < cfg.p_skip;
            const int inc = (x0 > 0 && skip8[(size_t)(y0 / 8) * w8 + (x0 - 1) / 8]) +
                            (y0 > 0 && skip8[(size_t)((y0 - 1) / 8) * w8 + x0 / 8]);
            E.decision(C.skip[inc], skip);
            fill(skip8, 8, w8, x0, y0, size, size, skip ? 1 : 0);
            if (skip) {
                fill(mode4, 4, p.W / 4, x0, y0, size, size, 1);
                prediction_unit(x0, y0, size, size, depth, true);
                return;
            }
            const bool intra = u01() < cfg.p_intra_cu;
            E.decision(C.pred_mode, intra);
            if (!intra) {
                inter_cu(x0, y0, log2, depth);
                return;
            }
        }
        const bool nxn = log2 == 3 && u01() < cfg.p_nxn;
        if (log2 == 3) E.decision(C.part_mode[0], nxn ? 0 : 1);   // part_mode: PART_2Nx2N = 1, PART_NxN = 0
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
        transform_tree(x0, y0, x0, y0, log2, 0, 0, nxn, max_depth, cmode, true, true, false);
    }

    // An inter CU: part_mode (9.3.3.7: "1" 2Nx2N; "01x" horizontal, "00x" vertical halves,
    // with AMP a context-coded "no AMP" bin (ctxInc 3) and a bypass bin for the quarter
    // side), its PUs, rqt_root_cbf (absent for a merged 2Nx2N PU), the transform tree.
    void inter_cu(int x0, int y0, int log2, int depth) {
        const int n = 1 << log2;
        const bool amp = p.amp && log2 > 3;
        // 0 2Nx2N, 1 2NxN, 2 Nx2N, 4 2NxnU, 5 2NxnD, 6 nLx2N, 7 nRx2N
        int pm = 0;
        if (u01() >= 0.4) {
            static const int with_amp[6] = {1, 2, 4, 5, 6, 7};
            pm = amp ? with_amp[uni(0, 5)] : uni(1, 2);
        }
        E.decision(C.part_mode[0], pm == 0);
        if (pm != 0) {
            const bool horizontal = pm == 1 || pm == 4 || pm == 5;
            E.decision(C.part_mode[1], horizontal);
            if (amp) {
                E.decision(C.part_mode[3], pm == 1 || pm == 2);
                if (pm >= 4) E.bypass(pm == 5 || pm == 7);
            }
        }
        fill(mode4, 4, p.W / 4, x0, y0, n, n, 1);
        int geo[2][4];   // PUs: x, y, w, h (relative)
        int npu = 2;
        switch (pm) {
        case 0: npu = 1; geo[0][0] = 0; geo[0][1] = 0; geo[0][2] = n; geo[0][3] = n; break;
        case 1: case 4: case 5: {
            const int h0 = pm == 1 ? n / 2 : (pm == 4 ? n / 4 : 3 * n / 4);
            const int a[2][4] = {{0, 0, n, h0}, {0, h0, n, n - h0}};
            std::memcpy(geo, a, sizeof(a));
            break;
        }
        default: {
            const int w0 = pm == 2 ? n / 2 : (pm == 6 ? n / 4 : 3 * n / 4);
            const int a[2][4] = {{0, 0, w0, n}, {w0, 0, n - w0, n}};
            std::memcpy(geo, a, sizeof(a));
            break;
        }
        }
        bool merge0 = false;
        for (int k = 0; k < npu; k++) {
            const bool m = prediction_unit(x0 + geo[k][0], y0 + geo[k][1], geo[k][2], geo[k][3], depth, false);
            if (k == 0) merge0 = m;
        }
        bool root = true;
        if (!(pm == 0 && merge0)) {
            root = u01() < 0.75;
            E.decision(C.rqt_root_cbf, root);
        }
        if (root) {
            const bool inter_split = p.depth_inter == 0 && pm != 0;   // interSplitFlag (7.4.9.8)
            transform_tree(x0, y0, x0, y0, log2, 0, 0, inter_split, p.depth_inter, -1, true, true, true);
        }
    }

    // Truncated unary with the first bin context-coded and the rest bypass (merge_idx,
    // cMax = MaxNumMergeCand - 1), or the first two context-coded (ref_idx_lX, 9.3.4.2.1).
    void truncated_unary(int v, int cmax, Ctx* ctx, int n_ctx) {
        for (int k = 0; k < cmax; k++) {
            const int bin = k < v;
            if (k < n_ctx) E.decision(ctx[k], bin);
            else E.bypass(bin);
            if (!bin) break;
        }
    }

    // k-th order Exp-Golomb, bypass bins (9.3.3.3)
    void exp_golomb(uint32_t v, int k) {
        while (v >= (1u << k)) {
            E.bypass(1);
            v -= 1u << k;
            k++;
        }
        E.bypass(0);
        while (k--) E.bypass((int)((v >> k) & 1u));
    }

    int draw_mvd() {
        if (u01() < 0.25) return 0;
        const int a = u01() < 0.7 ? uni(1, std::min(8, cfg.max_mvd)) : uni(1, cfg.max_mvd);
        return u01() < 0.5 ? -a : a;
    }

    // mvd_coding() (7.3.8.9): greater0 flags, greater1 flags, then per component
    // abs_mvd_minus2 (EG1) and the sign.
    void mvd_coding(int mx, int my) {
        const int a[2] = {std::abs(mx), std::abs(my)}, v[2] = {mx, my};
        for (int c = 0; c < 2; c++) E.decision(C.mvd_greater0, a[c] > 0);
        for (int c = 0; c < 2; c++)
            if (a[c] > 0) E.decision(C.mvd_greater1, a[c] > 1);
        for (int c = 0; c < 2; c++) {
            if (!a[c]) continue;
            if (a[c] > 1) exp_golomb((uint32_t)(a[c] - 2), 1);
            E.bypass(v[c] < 0);
        }
    }

    // prediction_unit() (7.3.8.6); returns merge_flag.  inter_pred_idc (9.3.3.x, 9.3.4.2.2):
    // "1" PRED_BI (context CtDepth), "00"/"01" PRED_L0/PRED_L1 (second bin context 4); a
    // PU with nPbW + nPbH = 12 has only the context-4 bin (no bi-prediction).
    bool prediction_unit(int x, int y, int w, int h, int depth, bool skip) {
        hevc_pu_t u{};
        u.x = (uint16_t)x;
        u.y = (uint16_t)y;
        u.w = (uint8_t)w;
        u.h = (uint8_t)h;
        u.wp = -1;
        const bool merge = skip || u01() < cfg.p_merge;
        if (!skip) E.decision(C.merge_flag, merge);
        if (merge) {
            if (max_merge > 1) truncated_unary(uni(0, max_merge - 1), max_merge - 1, &C.merge_idx, 1);
            u.ref_idx[0] = u.ref_idx[1] = -2;
            pus.push_back(u);
            return true;
        }
        int dir = 0;   // 0 PRED_L0, 1 PRED_L1, 2 PRED_BI
        if (slice_type == 0) {
            if (w + h != 12) {
                dir = uni(0, 2);
                E.decision(C.inter_pred_idc[depth], dir == 2);
                if (dir != 2) E.decision(C.inter_pred_idc[4], dir);
            } else {
                dir = uni(0, 1);
                E.decision(C.inter_pred_idc[4], dir);
            }
        }
        u.ref_idx[0] = u.ref_idx[1] = -1;
        for (int l = 0; l < 2; l++) {
            if (dir == 1 - l) continue;
            const int ref = uni(0, num_ref[l] - 1);
            if (num_ref[l] > 1) truncated_unary(ref, num_ref[l] - 1, C.ref_idx, 2);
            int mx = 0, my = 0;
            if (!(l == 1 && mvd_l1_zero && dir == 2)) {
                mx = draw_mvd();
                my = draw_mvd();
                mvd_coding(mx, my);
            }
            E.decision(C.mvp_flag, uni(0, 1));
            u.ref_idx[l] = (int8_t)ref;
            u.mv[l][0] = (int16_t)mx;
            u.mv[l][1] = (int16_t)my;
        }
        pus.push_back(u);
        return false;
    }

    void record(int c, int x, int y, int log2, int mode, bool coded, bool inter) {
        if (inter && !coded) return;   // a decoder sees the coded TUs of an inter CU only
        hevc_tu_t t{};
        t.x = (uint16_t)x;
        t.y = (uint16_t)y;
        t.log2_size = (uint8_t)log2;
        t.c_idx = (uint8_t)c;
        t.qp = (uint8_t)(c ? chroma_qp(qp) : qp);
        t.flags = (uint8_t)((inter ? 0 : HEVC_TU_INTRA) | (coded ? HEVC_TU_CODED : 0));
        t.intra_mode = (uint8_t)(inter ? 0 : mode);
        t.coeff_offset = 0;
        if (coded) {
            t.coeff_offset = (uint32_t)coeffs.size();
            coeffs.resize(coeffs.size() + ((size_t)1 << (2 * log2)), 0);
        }
        tus.push_back(t);
    }

    // transform_tree() (7.3.8.8) and transform_unit() (7.3.8.10).  nxn: IntraSplitFlag, or
    // interSplitFlag for an inter CU (both force the split at depth 0).  An inter CU's
    // cbf_luma at depth 0 is coded only when a chroma cbf is set (else it is 1).
    void transform_tree(int x0, int y0, int xb, int yb, int log2, int depth, int blk, bool nxn, int max_depth,
                        int cmode, bool parent_cb, bool parent_cr, bool inter) {
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
                               cb, cr, inter);
            return;
        }
        bool cbf_luma = true;
        if (!inter || depth != 0 || cb || cr) {
            cbf_luma = u01() < cfg.p_cbf;
            E.decision(C.cbf_luma[depth == 0 ? 1 : 0], cbf_luma);
        }
        const int w4 = p.W / 4;
        const int lmode = inter ? -1 : mode4[(size_t)(y0 / 4) * w4 + x0 / 4];
        record(0, x0, y0, log2, lmode, cbf_luma, inter);
        if (cbf_luma) residual(x0, y0, log2, 0, lmode);
        if (log2 > 2) {
            for (int c = 1; c <= 2; c++) {
                const bool f = c == 1 ? cb : cr;
                record(c, x0 / 2, y0 / 2, log2 - 1, cmode, f, inter);
                if (f) residual(x0 / 2, y0 / 2, log2 - 1, c, cmode);
            }
        } else if (blk == 3) {
            for (int c = 1; c <= 2; c++) {
                const bool f = c == 1 ? cb : cr;
                record(c, xb / 2, yb / 2, 2, cmode, f, inter);
                if (f) residual(xb / 2, yb / 2, 2, c, cmode);
            }
        }
    }

    void residual(int x0, int y0, int log2, int c, int mode);   // below

    // pred_weight_table() (7.3.6.3): denominators, then per list entry the flags and the
    // deltas of luma and chroma weights and offsets (within 7.4.7.3's ranges).
    void pred_weight_table(Bits& b) {
        const int lwd = uni(0, 7), cwd = uni(0, 7);
        b.ue((uint32_t)lwd);       // luma_log2_weight_denom
        b.se(cwd - lwd);           // delta_chroma_log2_weight_denom
        for (int l = 0; l < (slice_type == 0 ? 2 : 1); l++) {
            const int n = num_ref[l];
            bool lf[4], cf[4];
            for (int i = 0; i < n; i++) b.bit((lf[i] = u01() < 0.6) ? 1 : 0);   // luma_weight_lX_flag
            for (int i = 0; i < n; i++) b.bit((cf[i] = u01() < 0.5) ? 1 : 0);   // chroma_weight_lX_flag
            for (int i = 0; i < n; i++) {
                if (lf[i]) {
                    b.se(uni(-20, 20));   // delta_luma_weight_lX
                    b.se(uni(-30, 30));   // luma_offset_lX
                }
                if (cf[i])
                    for (int j = 0; j < 2; j++) {
                        b.se(uni(-20, 20));   // delta_chroma_weight_lX
                        b.se(uni(-60, 60));   // delta_chroma_offset_lX
                    }
            }
        }
    }

    // slice_segment_header() (7.3.6.1) and slice_segment_data() (7.3.8.1) of the picture's
    // one slice.  A P/B picture's short-term RPS (7.3.7, coded in the header) keeps the
    // pictures in gop.refs (most recent first, each used by this picture or not); both
    // reference lists repeat the used ones, most recent first (8.3.4, low delay).
    std::vector<uint8_t> slice_data_and_header(int poc, GopState& gop) {
        Bits b;
        const bool idr = slice_type == 2;
        b.bit(1);            // first_slice_segment_in_pic_flag
        if (idr) b.bit(0);   // no_output_of_prior_pics_flag
        b.ue(0);             // slice_pic_parameter_set_id
        b.ue((uint32_t)slice_type);
        int init_type = 0;
        if (!idr) {
            b.put((uint32_t)(poc & 255), 8);   // slice_pic_order_cnt_lsb
            b.bit(0);                          // short_term_ref_pic_set_sps_flag
            const int n = (int)gop.refs.size();
            std::vector<int> used((size_t)n);
            int n_used = 0;
            for (int i = 0; i < n; i++) n_used += used[(size_t)i] = (i == n - 1 && !n_used) || u01() < 0.7;
            b.ue((uint32_t)n);                 // num_negative_pics
            b.ue(0);                           // num_positive_pics
            int prev = poc;
            std::vector<int> cur;              // StCurrBefore
            for (int i = 0; i < n; i++) {
                b.ue((uint32_t)(prev - gop.refs[(size_t)i] - 1));   // delta_poc_s0_minus1
                b.bit(used[(size_t)i]);                              // used_by_curr_pic_s0_flag
                prev = gop.refs[(size_t)i];
                if (used[(size_t)i]) cur.push_back(gop.refs[(size_t)i]);
            }
            // the reference lists and the collocated picture
            const bool override_refs = u01() < 0.7;
            num_ref[0] = override_refs ? uni(1, 4) : 1;
            num_ref[1] = slice_type == 0 ? (override_refs ? uni(1, 4) : 1) : 0;
            bool tmvp = p.tmvp && u01() < 0.8;
            bool col_l0 = true;
            int col_ref = 0;
            if (tmvp) {
                col_l0 = slice_type == 1 || u01() < 0.5;
                const int nl = num_ref[col_l0 ? 0 : 1];
                std::vector<int> ok;   // entries after the last picture without TMVP (7.4.7.1)
                for (int i = 0; i < nl; i++)
                    if (cur[(size_t)i % cur.size()] >= gop.tmvp_barrier) ok.push_back(i);
                if (ok.empty()) tmvp = false;
                else col_ref = ok[(size_t)uni(0, (int)ok.size() - 1)];
            }
            if (!tmvp) gop.tmvp_barrier = poc;
            if (p.tmvp) b.bit(tmvp ? 1 : 0);   // slice_temporal_mvp_enabled_flag
            if (p.sao) {
                b.bit(1);    // slice_sao_luma_flag
                b.bit(1);    // slice_sao_chroma_flag
            }
            b.bit(override_refs ? 1 : 0);      // num_ref_idx_active_override_flag
            if (override_refs) {
                b.ue((uint32_t)(num_ref[0] - 1));
                if (slice_type == 0) b.ue((uint32_t)(num_ref[1] - 1));
            }
            if (slice_type == 0) {
                mvd_l1_zero = u01() < 0.3;
                b.bit(mvd_l1_zero ? 1 : 0);    // mvd_l1_zero_flag
            }
            const bool cabac_init = u01() < 0.3;
            b.bit(cabac_init ? 1 : 0);         // cabac_init_flag
            init_type = slice_type == 1 ? (cabac_init ? 2 : 1) : (cabac_init ? 1 : 2);
            if (tmvp) {
                if (slice_type == 0) b.bit(col_l0 ? 1 : 0);   // collocated_from_l0_flag
                if (num_ref[col_l0 ? 0 : 1] > 1) b.ue((uint32_t)col_ref);   // collocated_ref_idx
            }
            if (p.wp) pred_weight_table(b);
            max_merge = cfg.max_merge ? cfg.max_merge : uni(1, 5);
            b.ue((uint32_t)(5 - max_merge));   // five_minus_max_num_merge_cand
        } else if (p.sao) {
            b.bit(1);        // slice_sao_luma_flag
            b.bit(1);        // slice_sao_chroma_flag
        }
        b.se(qp - 26);       // slice_qp_delta
        b.bit(1);            // slice_loop_filter_across_slices_enabled_flag
        b.trailing();        // byte_alignment()
        // the pictures kept for the next picture: this one and the most recent others
        if (idr) gop.refs.clear();
        gop.refs.insert(gop.refs.begin(), poc);
        if ((int)gop.refs.size() > cfg.max_refs) gop.refs.resize((size_t)cfg.max_refs);
        C.init(init_type, qp);
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
// mode: the intra prediction mode of the block, -1 in an inter CU (diagonal scan).
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
    cfg->inter = 0;
    cfg->p_b = 0.5;
    cfg->max_refs = 2;
    cfg->p_intra_cu = 0.1;
    cfg->p_skip = 0.25;
    cfg->p_merge = 0.4;
    cfg->max_mvd = 64;
    cfg->amp = 1;
    cfg->tmvp = 1;
    cfg->max_merge = 0;
    cfg->wp = 0;
    cfg->depth_inter = 1;
}

hevcgen_stream_t* hevcgen_stream(const hevcgen_cfg_t* cfg) {
    if (!cfg || cfg->width <= 0 || cfg->height <= 0 || (cfg->width & 7) || (cfg->height & 7) || cfg->pictures < 1 ||
        cfg->log2_ctb < 4 || cfg->log2_ctb > 6 || cfg->max_level < 1 || cfg->qp_min < 0 || cfg->qp_max > 51 ||
        cfg->qp_min > cfg->qp_max || cfg->max_refs < 1 || cfg->max_refs > 4 || cfg->max_mvd < 1 ||
        cfg->max_mvd > 1 << 14 || cfg->max_merge < 0 || cfg->max_merge > 5 || cfg->depth_inter < 0 ||
        cfg->depth_inter > 2)
        return nullptr;
    std::mt19937_64 rng(cfg->seed);
    Params p{cfg->width, cfg->height, cfg->log2_ctb, cfg->sao ? 1 : 0};
    if (cfg->inter) {
        p.inter = 1;
        p.dpb_minus1 = cfg->max_refs;
        p.amp = cfg->amp ? 1 : 0;
        p.tmvp = cfg->tmvp ? 1 : 0;
        p.wp = cfg->wp ? 1 : 0;
    }
    p.depth_inter = cfg->depth_inter;
    std::vector<uint8_t> out;
    nal(out, 32, vps(p));
    nal(out, 33, sps(p));
    nal(out, 34, pps(p));
    auto* s = static_cast<hevcgen_stream_t*>(std::calloc(1, sizeof(hevcgen_stream_t)));
    s->pictures = cfg->pictures;
    s->num_tus = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->tus = static_cast<hevc_tu_t**>(std::calloc((size_t)cfg->pictures, sizeof(hevc_tu_t*)));
    s->num_coeffs = static_cast<uint64_t*>(std::calloc((size_t)cfg->pictures, sizeof(uint64_t)));
    s->coeffs = static_cast<int16_t**>(std::calloc((size_t)cfg->pictures, sizeof(int16_t*)));
    s->slice_type = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->num_pus = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->pus = static_cast<hevc_pu_t**>(std::calloc((size_t)cfg->pictures, sizeof(hevc_pu_t*)));
    GopState gop;
    for (int k = 0; k < cfg->pictures; k++) {
        Picture pic(*cfg, rng, p);
        pic.qp = std::uniform_int_distribution<int>(cfg->qp_min, cfg->qp_max)(rng);
        const bool idr = k == 0 || !cfg->inter;
        pic.slice_type = idr ? 2 : (std::uniform_real_distribution<double>(0.0, 1.0)(rng) < cfg->p_b ? 0 : 1);
        pic.wctb = (p.W + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
        pic.hctb = (p.H + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
        pic.depth8.assign((size_t)(p.W / 8) * (p.H / 8), 0);
        pic.skip8.assign((size_t)(p.W / 8) * (p.H / 8), 0);
        pic.mode4.assign((size_t)(p.W / 4) * (p.H / 4), 1);
        pic.coeffs.reserve((size_t)p.W * p.H * 3 / 2);
        nal(out, idr ? 19 : 1, pic.slice_data_and_header(idr ? 0 : k, gop));   // IDR_W_RADL or TRAIL_R
        s->slice_type[k] = pic.slice_type;
        s->num_pus[k] = (int32_t)pic.pus.size();
        s->pus[k] = static_cast<hevc_pu_t*>(std::malloc(sizeof(hevc_pu_t) * std::max<size_t>(1, pic.pus.size())));
        if (!pic.pus.empty())
            std::memcpy(s->pus[k], pic.pus.data(), sizeof(hevc_pu_t) * pic.pus.size());
        s->num_tus[k] = (int32_t)pic.tus.size();
        s->tus[k] = static_cast<hevc_tu_t*>(std::malloc(sizeof(hevc_tu_t) * std::max<size_t>(1, pic.tus.size())));
        if (!pic.tus.empty())
            std::memcpy(s->tus[k], pic.tus.data(), sizeof(hevc_tu_t) * pic.tus.size());
        s->num_coeffs[k] = pic.coeffs.size();
        s->coeffs[k] = static_cast<int16_t*>(std::malloc(sizeof(int16_t) * std::max<size_t>(1, pic.coeffs.size())));
        if (!pic.coeffs.empty())
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
        std::free(s->pus[k]);
    }
    std::free(s->slice_type);
    std::free(s->num_pus);
    std::free(s->pus);
    std::free(s->num_tus);
    std::free(s->tus);
    std::free(s->num_coeffs);
    std::free(s->coeffs);
    std::free(s->bytes);
    std::free(s);
}

}  // extern "C"
