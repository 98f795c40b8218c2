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
#include <functional>
#include <map>
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

// Annex B: start code, NAL unit header (nuh_layer_id 0, TemporalId tid), emulation prevention.
void nal(std::vector<uint8_t>& out, int type, const std::vector<uint8_t>& rbsp, int tid = 0) {
    const uint8_t sc[4] = {0, 0, 0, 1};
    out.insert(out.end(), sc, sc + 4);
    out.push_back((uint8_t)(type << 1));
    out.push_back((uint8_t)(tid + 1));   // nuh_temporal_id_plus1
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

// Where each RBSP byte lands in the NAL unit payload once nal() inserts the emulation
// prevention bytes (7.4.2): entry point offsets count payload bytes.
std::vector<size_t> nal_positions(const std::vector<uint8_t>& rbsp) {
    std::vector<size_t> pos(rbsp.size() + 1);
    size_t o = 0;
    int zeros = 0;
    for (size_t i = 0; i < rbsp.size(); i++) {
        if (zeros >= 2 && rbsp[i] <= 3) {
            o++;
            zeros = 0;
        }
        pos[i] = o++;
        zeros = rbsp[i] == 0 ? zeros + 1 : 0;
    }
    pos[rbsp.size()] = o;
    return pos;
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
// cu_qp_delta_abs (2), cu_transquant_bypass_flag (1), transform_skip_flag (luma, chroma):
// the same values for every initType
const uint8_t kInitQpDelta = 154, kInitBypass = 154, kInitTskip = 139;

struct Contexts {
    Ctx sao_merge, sao_type, split_cu[3], skip[3], pred_mode, part_mode[4], prev_intra_luma, intra_chroma, rqt_root_cbf,
        merge_flag, merge_idx, inter_pred_idc[5], ref_idx[2], mvp_flag, mvd_greater0, mvd_greater1, split_transform[3],
        cbf_luma[2], cbf_chroma[4], last_x[18], last_y[18], csbf[4], sig[42], greater1[24], greater2[6], qp_delta[2],
        bypass, tskip[2];
    void init(int t, int qp) {   // t: initType
        for (int i = 0; i < 2; i++) qp_delta[i].init(kInitQpDelta, qp);
        bypass.init(kInitBypass, qp);
        for (int i = 0; i < 2; i++) tskip[i].init(kInitTskip, qp);
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
void profile_tier_level(Bits& b, int max_sub_layers_minus1) {
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
    for (int i = 0; i < max_sub_layers_minus1; i++) {
        b.bit(0);          // sub_layer_profile_present_flag
        b.bit(0);          // sub_layer_level_present_flag
    }
    if (max_sub_layers_minus1 > 0)
        for (int i = max_sub_layers_minus1; i < 8; i++) b.put(0, 2);   // reserved_zero_2bits
}

// A short-term RPS as deltas to the current POC: before it (closest first) and after it
// (closest first), each with used_by_curr_pic.
struct Rps {
    std::vector<int> d0, d1, u0, u1;
    bool operator==(const Rps& o) const { return d0 == o.d0 && d1 == o.d1 && u0 == o.u0 && u1 == o.u1; }
};

// st_ref_pic_set(idx) (7.3.7) of t.  With idx > 0 it is predicted from a set of sets[]
// (inter_ref_pic_set_prediction_flag) when some deltaRps makes every entry of t a
// candidate (7.4.8: each entry of the reference set moved by deltaRps, and deltaRps
// itself); the derivation then lists them in t's order.  In a slice header (idx equal to
// the number of SPS sets) any SPS set may be the reference, through delta_idx_minus1.
void st_ref_pic_set(Bits& b, const Rps& t, int idx, const std::vector<Rps>& sets, bool in_slice, std::mt19937_64& rng) {
    auto uni = [&](int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); };
    if (idx != 0) {
        bool predicted = false;
        if (uni(0, 9) < 7) {
            const int ref = in_slice ? uni(0, idx - 1) : idx - 1;
            const Rps& r = sets[(size_t)ref];
            std::vector<int> cand(r.d0);   // j = 0 .. NumDeltaPocs: S0, S1, then deltaRps itself
            cand.insert(cand.end(), r.d1.begin(), r.d1.end());
            std::vector<int> deltas;
            for (int d = -16; d <= 16; d++)
                if (d) deltas.push_back(d);
            std::shuffle(deltas.begin(), deltas.end(), rng);
            for (int drps : deltas) {
                auto used_of = [&](int v) -> int {   // -1: not in t
                    for (size_t i = 0; i < t.d0.size(); i++)
                        if (t.d0[i] == v) return t.u0[i];
                    for (size_t i = 0; i < t.d1.size(); i++)
                        if (t.d1[i] == v) return t.u1[i];
                    return -1;
                };
                size_t covered = 0;
                for (size_t j = 0; j <= cand.size(); j++) {
                    const int v = j < cand.size() ? cand[j] + drps : drps;
                    covered += v != 0 && used_of(v) >= 0;
                }
                if (covered != t.d0.size() + t.d1.size()) continue;
                b.bit(1);                                        // inter_ref_pic_set_prediction_flag
                if (in_slice) b.ue((uint32_t)(idx - 1 - ref));   // delta_idx_minus1
                b.bit(drps < 0 ? 1 : 0);                         // delta_rps_sign
                b.ue((uint32_t)(std::abs(drps) - 1));            // abs_delta_rps_minus1
                for (size_t j = 0; j <= cand.size(); j++) {
                    const int v = j < cand.size() ? cand[j] + drps : drps;
                    const int u = v != 0 ? used_of(v) : -1;
                    b.bit(u == 1 ? 1 : 0);                       // used_by_curr_pic_flag
                    if (u != 1) b.bit(u == 0 ? 1 : 0);           // use_delta_flag
                }
                predicted = true;
                break;
            }
        }
        if (predicted) return;
        b.bit(0);                                                // inter_ref_pic_set_prediction_flag
    }
    b.ue((uint32_t)t.d0.size());                                 // num_negative_pics
    b.ue((uint32_t)t.d1.size());                                 // num_positive_pics
    int prev = 0;
    for (size_t i = 0; i < t.d0.size(); i++) {
        b.ue((uint32_t)(prev - t.d0[i] - 1));                    // delta_poc_s0_minus1
        b.bit(t.u0[i]);                                          // used_by_curr_pic_s0_flag
        prev = t.d0[i];
    }
    prev = 0;
    for (size_t i = 0; i < t.d1.size(); i++) {
        b.ue((uint32_t)(t.d1[i] - prev - 1));                    // delta_poc_s1_minus1
        b.bit(t.u1[i]);                                          // used_by_curr_pic_s1_flag
        prev = t.d1[i];
    }
}

// The stream's parameter sets: what the SPS and PPS enable, drawn once per stream.
struct Params {
    int W, H, log2_ctb, sao;
    int inter = 0, dpb_minus1 = 1, num_reorder = 0, amp = 0, tmvp = 0, wp = 0, depth_inter = 1, log2_pml = 2;
    int qp_delta = 0, qp_delta_depth = 0;                       // cu_qp_delta_enabled_flag, diff_cu_qp_delta_depth
    int cb_qp_offset = 0, cr_qp_offset = 0, slice_chroma_offsets = 0;
    int dbk_ctl = 0, dbk_override = 0, dbk_disabled = 0, beta_div2 = 0, tc_div2 = 0;
    int lf_across_slices = 1, dependent_slices = 0;
    int bypass = 0, tskip = 0, sdh = 0;
    int pcm = 0, pcm_bits_y = 8, pcm_bits_c = 8, pcm_log2_min = 3, pcm_log2_max = 3, pcm_lf_disabled = 0;
    int scaling = 0;                                            // 0 off, 1 default lists, 2 SPS lists, 3 PPS lists
    int crop[4] = {0, 0, 0, 0};                                 // conformance window offsets (chroma units)
    int output_flag = 0;                                        // output_flag_present_flag
    int long_term = 0;                                          // long_term_ref_pics_present_flag
    int list_mod = 0;                                           // lists_modification_present_flag
    int poc_bits = 8;                                           // log2_max_pic_order_cnt_lsb
    int bit_depth = 8;                                          // BitDepthY = BitDepthC
    int max_tid = 0;                                            // sps_max_sub_layers_minus1
    int extra = 0;             // AUD, SEI, filler, EOS/EOB NAL units, VUI, slice_reserved_flag, header extensions
    int extra_bits = 0;                                         // num_extra_slice_header_bits
    int pps_id = 0;                                             // pps_pic_parameter_set_id
    std::vector<Rps> rps_sets;                                  // the SPS's st_ref_pic_set()s
    int wpp = 0;                                                // entropy_coding_sync_enabled_flag
    std::vector<int> col_bd, row_bd;                            // tile boundaries in CTBs (one tile: {0, w})
    int uniform_tiles = 0, lf_across_tiles = 1;
    int log2_max_tb() const { return std::min(5, log2_ctb); }
    int tiles() const { return (int)(col_bd.size() - 1) * (int)(row_bd.size() - 1); }
};

// scaling_list_data() (7.3.4): per size and matrix, a reference to an earlier (or the
// default) list, or the list itself as DPCM deltas (every ScalingList entry 1..255).
void scaling_list_data(Bits& b, std::mt19937_64& rng) {
    auto uni = [&](int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); };
    for (int size_id = 0; size_id < 4; size_id++)
        for (int matrix_id = 0; matrix_id < 6; matrix_id += size_id == 3 ? 3 : 1) {
            const bool explicit_list = uni(0, 2) != 0;
            b.bit(explicit_list ? 1 : 0);                      // scaling_list_pred_mode_flag
            if (!explicit_list) {
                b.ue((uint32_t)uni(0, size_id == 3 ? matrix_id / 3 : matrix_id));   // ..._pred_matrix_id_delta
                continue;
            }
            int next = 8;
            const int n = std::min(64, 1 << (4 + (size_id << 1)));
            if (size_id > 1) {
                const int dc = uni(1, 255);
                b.se(dc - 8);                                  // scaling_list_dc_coef_minus8
                next = dc;
            }
            for (int i = 0; i < n; i++) {
                const int v = uni(0, 3) ? uni(8, 40) : uni(1, 255);
                const int delta = ((v - next + 128) & 255) - 128;
                b.se(delta);                                   // scaling_list_delta_coef
                next = v;
            }
        }
}

std::vector<uint8_t> vps(const Params& p) {
    Bits b;
    b.put(0, 4);           // vps_video_parameter_set_id
    b.bit(1);              // vps_base_layer_internal_flag
    b.bit(1);              // vps_base_layer_available_flag
    b.put(0, 6);           // vps_max_layers_minus1
    b.put((uint32_t)p.max_tid, 3);           // vps_max_sub_layers_minus1
    b.bit(p.max_tid == 0 ? 1 : 0);           // vps_temporal_id_nesting_flag
    b.put(0xFFFF, 16);     // vps_reserved_0xffff_16bits
    profile_tier_level(b, p.max_tid);
    b.bit(1);              // vps_sub_layer_ordering_info_present_flag
    for (int i = 0; i <= p.max_tid; i++) {   // the same for every sub-layer
        b.ue((uint32_t)p.dpb_minus1);        // vps_max_dec_pic_buffering_minus1
        b.ue((uint32_t)p.num_reorder);       // vps_max_num_reorder_pics
        b.ue(0);                             // vps_max_latency_increase_plus1
    }
    b.put(0, 6);           // vps_max_layer_id
    b.ue(0);               // vps_num_layer_sets_minus1
    b.bit(0);              // vps_timing_info_present_flag
    b.bit(0);              // vps_extension_flag
    b.trailing();
    return b.buf;
}

// vui_parameters() (E.2.1) with fields drawn; no HRD parameters, progressive frames
// (field_seq_flag 0, as general_frame_only_constraint_flag requires), motion vectors over
// picture boundaries allowed.
void vui_parameters(Bits& b, std::mt19937_64& rng) {
    auto uni = [&](int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); };
    const bool ar = uni(0, 1);
    b.bit(ar);                                   // aspect_ratio_info_present_flag
    if (ar) {
        const int idc = uni(0, 1) ? 255 : uni(0, 16);
        b.put((uint32_t)idc, 8);                 // aspect_ratio_idc
        if (idc == 255) {
            b.put((uint32_t)uni(1, 65535), 16);  // sar_width
            b.put((uint32_t)uni(1, 65535), 16);  // sar_height
        }
    }
    const bool ov = uni(0, 1);
    b.bit(ov);                                   // overscan_info_present_flag
    if (ov) b.bit(uni(0, 1));                    // overscan_appropriate_flag
    const bool vs = uni(0, 1);
    b.bit(vs);                                   // video_signal_type_present_flag
    if (vs) {
        b.put((uint32_t)uni(0, 5), 3);           // video_format
        b.bit(uni(0, 1));                        // video_full_range_flag
        const bool cd = uni(0, 1);
        b.bit(cd);                               // colour_description_present_flag
        if (cd) {
            b.put((uint32_t)uni(1, 12), 8);      // colour_primaries
            b.put((uint32_t)uni(1, 18), 8);      // transfer_characteristics
            b.put((uint32_t)uni(0, 11), 8);      // matrix_coeffs
        }
    }
    const bool cl = uni(0, 1);
    b.bit(cl);                                   // chroma_loc_info_present_flag
    if (cl) {
        b.ue((uint32_t)uni(0, 5));               // chroma_sample_loc_type_top_field
        b.ue((uint32_t)uni(0, 5));               // chroma_sample_loc_type_bottom_field
    }
    b.bit(0);                                    // neutral_chroma_indication_flag
    b.bit(0);                                    // field_seq_flag
    b.bit(0);                                    // frame_field_info_present_flag
    const bool dw = uni(0, 1);
    b.bit(dw);                                   // default_display_window_flag
    if (dw)
        for (int k = 0; k < 4; k++) b.ue((uint32_t)uni(0, 4));   // def_disp_win_*_offset
    const bool ti = uni(0, 1);
    b.bit(ti);                                   // vui_timing_info_present_flag
    if (ti) {
        b.put(1001, 32);                         // vui_num_units_in_tick
        b.put(60000, 32);                        // vui_time_scale
        const bool pp = uni(0, 1);
        b.bit(pp);                               // vui_poc_proportional_to_timing_flag
        if (pp) b.ue(0);                         // vui_num_ticks_poc_diff_one_minus1
        b.bit(0);                                // vui_hrd_parameters_present_flag
    }
    const bool br = uni(0, 1);
    b.bit(br);                                   // bitstream_restriction_flag
    if (br) {
        b.bit(0);                                // tiles_fixed_structure_flag
        b.bit(1);                                // motion_vectors_over_pic_boundaries_flag
        b.bit(0);                                // restricted_ref_pic_lists_flag
        b.ue(0);                                 // min_spatial_segmentation_idc
        b.ue(0);                                 // max_bytes_per_pic_denom
        b.ue(0);                                 // max_bits_per_min_cu_denom
        b.ue(15);                                // log2_max_mv_length_horizontal
        b.ue(15);                                // log2_max_mv_length_vertical
    }
}

std::vector<uint8_t> sps(const Params& p, std::mt19937_64& rng) {
    Bits b;
    b.put(0, 4);           // sps_video_parameter_set_id
    b.put((uint32_t)p.max_tid, 3);           // sps_max_sub_layers_minus1
    b.bit(p.max_tid == 0 ? 1 : 0);           // sps_temporal_id_nesting_flag
    profile_tier_level(b, p.max_tid);
    b.ue(0);               // sps_seq_parameter_set_id
    b.ue(1);               // chroma_format_idc: 4:2:0
    b.ue((uint32_t)p.W);   // pic_width_in_luma_samples
    b.ue((uint32_t)p.H);   // pic_height_in_luma_samples
    b.bit(p.crop[0] | p.crop[1] | p.crop[2] | p.crop[3] ? 1 : 0);   // conformance_window_flag
    if (p.crop[0] | p.crop[1] | p.crop[2] | p.crop[3])
        for (int k = 0; k < 4; k++) b.ue((uint32_t)p.crop[k]);   // conf_win_left/right/top/bottom_offset
    b.ue((uint32_t)(p.bit_depth - 8));       // bit_depth_luma_minus8
    b.ue((uint32_t)(p.bit_depth - 8));       // bit_depth_chroma_minus8
    b.ue((uint32_t)(p.poc_bits - 4));        // log2_max_pic_order_cnt_lsb_minus4
    b.bit(1);              // sps_sub_layer_ordering_info_present_flag
    for (int i = 0; i <= p.max_tid; i++) {
        b.ue((uint32_t)p.dpb_minus1);        // sps_max_dec_pic_buffering_minus1
        b.ue((uint32_t)p.num_reorder);       // sps_max_num_reorder_pics
        b.ue(0);                             // sps_max_latency_increase_plus1
    }
    b.ue(0);               // log2_min_luma_coding_block_size_minus3: 8x8
    b.ue((uint32_t)(p.log2_ctb - 3));        // log2_diff_max_min_luma_coding_block_size
    b.ue(0);               // log2_min_luma_transform_block_size_minus2: 4x4
    b.ue((uint32_t)(p.log2_max_tb() - 2));   // log2_diff_max_min_luma_transform_block_size
    b.ue((uint32_t)p.depth_inter);           // max_transform_hierarchy_depth_inter
    b.ue(1);               // max_transform_hierarchy_depth_intra
    b.bit(p.scaling ? 1 : 0);                // scaling_list_enabled_flag
    if (p.scaling) {
        b.bit(p.scaling == 2 ? 1 : 0);       // sps_scaling_list_data_present_flag
        if (p.scaling == 2) scaling_list_data(b, rng);
    }
    b.bit(p.amp ? 1 : 0);  // amp_enabled_flag
    b.bit(p.sao ? 1 : 0);  // sample_adaptive_offset_enabled_flag
    b.bit(p.pcm ? 1 : 0);  // pcm_enabled_flag
    if (p.pcm) {
        b.put((uint32_t)(p.pcm_bits_y - 1), 4);              // pcm_sample_bit_depth_luma_minus1
        b.put((uint32_t)(p.pcm_bits_c - 1), 4);              // pcm_sample_bit_depth_chroma_minus1
        b.ue((uint32_t)(p.pcm_log2_min - 3));                // log2_min_pcm_luma_coding_block_size_minus3
        b.ue((uint32_t)(p.pcm_log2_max - p.pcm_log2_min));   // log2_diff_max_min_pcm_luma_coding_block_size
        b.bit(p.pcm_lf_disabled ? 1 : 0);                    // pcm_loop_filter_disabled_flag
    }
    b.ue((uint32_t)p.rps_sets.size());       // num_short_term_ref_pic_sets
    for (size_t i = 0; i < p.rps_sets.size(); i++) st_ref_pic_set(b, p.rps_sets[i], (int)i, p.rps_sets, false, rng);
    b.bit(p.long_term ? 1 : 0);              // long_term_ref_pics_present_flag
    if (p.long_term) b.ue(0);                // num_long_term_ref_pics_sps
    b.bit(p.tmvp ? 1 : 0); // sps_temporal_mvp_enabled_flag
    b.bit(1);              // strong_intra_smoothing_enabled_flag
    b.bit(p.extra ? 1 : 0);  // vui_parameters_present_flag
    if (p.extra) vui_parameters(b, rng);
    b.bit(0);              // sps_extension_present_flag
    b.trailing();
    return b.buf;
}

std::vector<uint8_t> pps(const Params& p, std::mt19937_64& rng) {
    Bits b;
    b.ue((uint32_t)p.pps_id);                // pps_pic_parameter_set_id
    b.ue(0);               // pps_seq_parameter_set_id
    b.bit(p.dependent_slices ? 1 : 0);       // dependent_slice_segments_enabled_flag
    b.bit(p.output_flag ? 1 : 0);             // output_flag_present_flag
    b.put((uint32_t)p.extra_bits, 3);        // num_extra_slice_header_bits
    b.bit(p.sdh ? 1 : 0);  // sign_data_hiding_enabled_flag
    b.bit(p.inter ? 1 : 0);   // cabac_init_present_flag (cabac_init_flag drawn per slice)
    b.ue(0);               // num_ref_idx_l0_default_active_minus1
    b.ue(0);               // num_ref_idx_l1_default_active_minus1
    b.se(0);               // init_qp_minus26
    b.bit(0);              // constrained_intra_pred_flag
    b.bit(p.tskip ? 1 : 0);                  // transform_skip_enabled_flag
    b.bit(p.qp_delta ? 1 : 0);               // cu_qp_delta_enabled_flag
    if (p.qp_delta) b.ue((uint32_t)p.qp_delta_depth);   // diff_cu_qp_delta_depth
    b.se(p.cb_qp_offset);  // pps_cb_qp_offset
    b.se(p.cr_qp_offset);  // pps_cr_qp_offset
    b.bit(p.slice_chroma_offsets ? 1 : 0);   // pps_slice_chroma_qp_offsets_present_flag
    b.bit(p.wp ? 1 : 0);   // weighted_pred_flag
    b.bit(p.wp ? 1 : 0);   // weighted_bipred_flag
    b.bit(p.bypass ? 1 : 0);                 // transquant_bypass_enabled_flag
    const bool tiles = p.tiles() > 1;
    b.bit(tiles ? 1 : 0);  // tiles_enabled_flag
    b.bit(p.wpp ? 1 : 0);  // entropy_coding_sync_enabled_flag
    if (tiles) {
        const int nc = (int)p.col_bd.size() - 1, nr = (int)p.row_bd.size() - 1;
        b.ue((uint32_t)(nc - 1));            // num_tile_columns_minus1
        b.ue((uint32_t)(nr - 1));            // num_tile_rows_minus1
        b.bit(p.uniform_tiles ? 1 : 0);      // uniform_spacing_flag
        if (!p.uniform_tiles) {
            for (int i = 0; i < nc - 1; i++) b.ue((uint32_t)(p.col_bd[(size_t)i + 1] - p.col_bd[(size_t)i] - 1));
            for (int i = 0; i < nr - 1; i++) b.ue((uint32_t)(p.row_bd[(size_t)i + 1] - p.row_bd[(size_t)i] - 1));
        }
        b.bit(p.lf_across_tiles ? 1 : 0);    // loop_filter_across_tiles_enabled_flag
    }
    b.bit(p.lf_across_slices ? 1 : 0);       // pps_loop_filter_across_slices_enabled_flag
    b.bit(p.dbk_ctl ? 1 : 0);                // deblocking_filter_control_present_flag
    if (p.dbk_ctl) {
        b.bit(p.dbk_override ? 1 : 0);       // deblocking_filter_override_enabled_flag
        b.bit(p.dbk_disabled ? 1 : 0);       // pps_deblocking_filter_disabled_flag
        if (!p.dbk_disabled) {
            b.se(p.beta_div2);               // pps_beta_offset_div2
            b.se(p.tc_div2);                 // pps_tc_offset_div2
        }
    }
    b.bit(p.scaling == 3 ? 1 : 0);           // pps_scaling_list_data_present_flag
    if (p.scaling == 3) scaling_list_data(b, rng);
    b.bit(p.list_mod ? 1 : 0);               // lists_modification_present_flag
    b.ue((uint32_t)(p.log2_pml - 2));        // log2_parallel_merge_level_minus2
    b.bit(p.extra ? 1 : 0);                  // slice_segment_header_extension_present_flag
    b.bit(0);              // pps_extension_present_flag
    b.trailing();
    return b.buf;
}

// chroma Qp' of 4:2:0 (8.6.1, table 8-10) for the records: qPi clipped to
// -QpBdOffsetC..57, mapped, plus QpBdOffsetC (bd_off)
int chroma_qp(int qpi, int bd_off) {
    static const int tab[14] = {29, 30, 31, 32, 33, 33, 34, 34, 35, 35, 36, 36, 37, 37};
    qpi = std::min(57, std::max(-bd_off, qpi));
    return (qpi < 30 ? qpi : (qpi > 43 ? qpi - 6 : tab[qpi - 30])) + bd_off;
}

}  // namespace

namespace {

// ---- one picture ----------------------------------------------------------------------------
// The reference picture state carried from one picture to the next.
// One picture of the coded sequence, planned before any is coded: its POC, slice type and
// decode index, and its short-term RPS (7.4.8): the pictures kept, those before it in output
// order (closest first) and those after it (closest first), each used by it or not.
struct PicPlan {
    int poc = 0, slice_type = 2, decode_idx = 0, nal_type = 19, tid = 0;   // tid: TemporalId
    bool output = true, no_output_of_prior = false;   // pic_output_flag, no_output_of_prior_pics_flag
    std::vector<int> neg, pos, lt;   // lt: POCs kept as long-term reference pictures
    std::vector<int> neg_used, pos_used, lt_used, lt_msb;   // lt_msb: delta_poc_msb_present_flag
};

Rps rps_of(const PicPlan& pl) {
    Rps r;
    for (size_t i = 0; i < pl.neg.size(); i++) {
        r.d0.push_back(pl.neg[i] - pl.poc);
        r.u0.push_back(pl.neg_used[i]);
    }
    for (size_t i = 0; i < pl.pos.size(); i++) {
        r.d1.push_back(pl.pos[i] - pl.poc);
        r.u1.push_back(pl.pos_used[i]);
    }
    return r;
}

// State carried from one picture to the next: each coded POC's decode index, and the decode
// index of the last picture whose slice_temporal_mvp_enabled_flag was 0 (7.4.7.1: later
// pictures take no collocated picture decoded before it).
struct GopState {
    std::vector<int> decode_idx_of_poc;
    int tmvp_barrier = 0;
};

struct Picture {
    const hevcgen_cfg_t& cfg;
    std::mt19937_64& rng;
    Params p;
    int wctb = 0, hctb = 0;
    // the picture's slices and tiles: per raster CTB address, the SliceAddrRs of its slice
    // and its TileId; CtbAddrTsToRs
    std::vector<int> ctb_slice, ctb_tile, ts_to_rs;
    int cur_slice = 0, cur_tile = 0;
    // the slice: type (0 B, 1 P, 2 I), SliceQpY, chroma QP offsets (PPS + slice), SAO
    // flags, active reference list sizes, MaxNumMergeCand
    int slice_type = 2, qp = 26, cb_off = 0, cr_off = 0;
    bool sao_luma = true, sao_chroma = true;
    int num_ref[2] = {0, 0}, max_merge = 5;
    bool mvd_l1_zero = false;
    // quantization groups (8.6.1): QpY per 8x8 unit, the last CU's QpY, the current group
    std::vector<uint8_t> qp8;
    int last_cu_qp = 26, qg_x = 0, qg_y = 0, qg_pred = 26, qp_delta_val = 0;
    bool first_qg = true, qg_new = false, qp_delta_coded = false;
    bool cu_bypass = false;   // cu_transquant_bypass_flag of the current CU
    bool pcm_cu = false;      // pcm_flag of the current CU
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

    // z-scan availability of a neighbouring luma location (6.4.1): inside the picture, in
    // the current slice and tile (left and above neighbours there are decoded already)
    bool avail(int xN, int yN) const {
        if (xN < 0 || yN < 0 || xN >= p.W || yN >= p.H) return false;
        const size_t a = (size_t)(yN >> p.log2_ctb) * (size_t)wctb + (size_t)(xN >> p.log2_ctb);
        return ctb_slice[a] == cur_slice && ctb_tile[a] == cur_tile;
    }

    // QpY of the current CU (8.6.1): the group's prediction plus CuQpDeltaVal
    int cu_qp() const { return p.qp_delta ? (qg_pred + qp_delta_val + 52) % 52 : qp; }

    // qPY_PRED of a new quantization group at (qg_x, qg_y): the left and above groups'
    // QpY when they lie in the same CTB, else qPY_PREV (the previous CU's QpY, or SliceQpY
    // for the first group of a slice, a tile, or a CTB row under WPP)
    void start_quantization_group() {
        const int prev = first_qg ? qp : last_cu_qp;
        first_qg = false;
        const int w8 = p.W / 8, mask = (1 << p.log2_ctb) - 1;
        const int qa = (qg_x & mask) ? qp8[(size_t)(qg_y / 8) * w8 + (qg_x - 1) / 8] : prev;
        const int qb = (qg_y & mask) ? qp8[(size_t)((qg_y - 1) / 8) * w8 + qg_x / 8] : prev;
        qg_pred = (qa + qb + 1) >> 1;
    }

    // coding_quadtree() (7.3.8.4); split_cu_flag context: available neighbours deeper than
    // this node (9.3.4.2.2).  A node of the quantization group size or larger starts a
    // group (IsCuQpDeltaCoded = 0, CuQpDeltaVal = 0).
    void coding_quadtree(int x0, int y0, int log2, int depth) {
        const int size = 1 << log2;
        if (p.qp_delta && log2 >= p.log2_ctb - p.qp_delta_depth) {
            qp_delta_coded = false;
            qp_delta_val = 0;
            qg_x = x0;
            qg_y = y0;
            qg_new = true;
        }
        bool split;
        if (x0 + size <= p.W && y0 + size <= p.H && log2 > 3) {
            split = u01() < cfg.p_split;
            const int w8 = p.W / 8;
            const int inc = (avail(x0 - 1, y0) && depth8[(size_t)(y0 / 8) * w8 + (x0 - 1) / 8] > depth) +
                            (avail(x0, y0 - 1) && depth8[(size_t)((y0 - 1) / 8) * w8 + x0 / 8] > depth);
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
        if (qg_new || !p.qp_delta) {
            if (p.qp_delta) start_quantization_group();
            qg_new = false;
        }
        pcm_cu = false;
        coding_unit(x0, y0, log2, depth);
        if (!(pcm_cu && (cfg.ref_quirks & HEVCGEN_QUIRK_TILES_PCM))) last_cu_qp = cu_qp();
        fill(qp8, 8, w8, x0, y0, size, size, (uint8_t)last_cu_qp);
    }

    // fill a per-unit map over a rectangle of luma samples
    static void fill(std::vector<uint8_t>& m, int unit, int stride, int x0, int y0, int w, int h, uint8_t v) {
        for (int y = y0 / unit; y < (y0 + h) / unit; y++)
            for (int x = x0 / unit; x < (x0 + w) / unit; x++) m[(size_t)y * stride + x] = v;
    }

    // candModeList of a prediction block (8.4.2)
    void mpm(int xPb, int yPb, int cand[3]) {
        const int w4 = p.W / 4;
        const int a = avail(xPb - 1, yPb) ? mode4[(size_t)(yPb / 4) * w4 + (xPb - 1) / 4] : 1;
        const bool above_in_ctb_row = yPb - 1 >= ((yPb >> p.log2_ctb) << p.log2_ctb);
        const int b = (avail(xPb, yPb - 1) && above_in_ctb_row) ? mode4[(size_t)((yPb - 1) / 4) * w4 + xPb / 4] : 1;
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
        cu_bypass = false;
        if (p.bypass) {
            cu_bypass = u01() < cfg.p_bypass;
            E.decision(C.bypass, cu_bypass);   // cu_transquant_bypass_flag
        }
        if (slice_type != 2) {
            const int w8 = p.W / 8;
            const bool skip = u01() < cfg.p_skip;
            const int inc = (avail(x0 - 1, y0) && skip8[(size_t)(y0 / 8) * w8 + (x0 - 1) / 8]) +
                            (avail(x0, y0 - 1) && skip8[(size_t)((y0 - 1) / 8) * w8 + x0 / 8]);
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
        if (!nxn && p.pcm && log2 >= p.pcm_log2_min && log2 <= p.pcm_log2_max) {
            const bool pcm = u01() < cfg.p_pcm;
            E.terminate(pcm);   // pcm_flag
            if (pcm) {
                pcm_sample(x0, y0, log2);
                return;
            }
        }
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

    // cu_qp_delta_abs (9.3.3.10: prefix TR cMax 5, first bin context 0, the others context
    // 1; suffix EG0 bypass) and cu_qp_delta_sign_flag; CuQpDeltaVal in -26..25 (7.4.9.14)
    void cu_qp_delta() {
        int v = u01() < 0.6 ? uni(-3, 3) : uni(-26, 25);
        // above 8 bits QpY stays in 0..51, where the wrap of 8.6.1 never applies (the
        // records' QP is unsigned)
        if (p.bit_depth > 8) v = std::min(51 - qg_pred, std::max(-qg_pred, v));
        const int a = std::abs(v);
        for (int k = 0; k < 5; k++) {
            E.decision(C.qp_delta[k ? 1 : 0], k < a);
            if (k >= a) break;
        }
        if (a >= 5) exp_golomb((uint32_t)(a - 5), 0);
        if (a) E.bypass(v < 0);
        qp_delta_val = v;
        qp_delta_coded = true;
    }

    // pcm_sample() (7.3.8.7) after a pcm_flag of 1: the arithmetic code is flushed (the
    // terminate bin's flush ends in a 1 bit), pcm_alignment_zero_bits, the samples at
    // PcmBitDepth bits, then the arithmetic encoder restarts (9.3.2.5).  The records: one
    // PCM TU per plane whose levels are the reconstructed samples (value << (8 - depth)).
    void pcm_sample(int x0, int y0, int log2) {
        pcm_cu = true;
        Bits& b = *E.out;
        if ((cfg.ref_quirks & HEVCGEN_QUIRK_TILES_PCM) && b.n == 0) b.put(0x80, 8);
        b.align_zero();
        fill(mode4, 4, p.W / 4, x0, y0, 1 << log2, 1 << log2, 1);
        for (int c = 0; c < 3; c++) {
            const int l2 = c ? log2 - 1 : log2, bits = c ? p.pcm_bits_c : p.pcm_bits_y;
            hevc_tu_t t{};
            t.x = (uint16_t)(c ? x0 / 2 : x0);
            t.y = (uint16_t)(c ? y0 / 2 : y0);
            t.log2_size = (uint8_t)l2;
            t.c_idx = (uint8_t)c;
            t.qp = (uint8_t)(cu_qp() + 6 * (p.bit_depth - 8));
            t.flags = (uint8_t)(HEVC_TU_INTRA | HEVC_TU_CODED | HEVC_TU_PCM | (cu_bypass ? HEVC_TU_BYPASS : 0));
            t.intra_mode = 1;
            t.coeff_offset = (uint32_t)coeffs.size();
            for (int i = 0; i < 1 << (2 * l2); i++) {
                const int v = uni(0, (1 << bits) - 1);
                b.put((uint32_t)v, bits);
                coeffs.push_back((int16_t)(v << (p.bit_depth - bits)));
            }
            tus.push_back(t);
        }
        E.start(&b);
        if (cfg.ref_quirks & HEVCGEN_QUIRK_TILES_PCM) C.init(init_type, qp);
    }

    void record(int c, int x, int y, int log2, int mode, bool coded, bool inter) {
        if (inter && !coded) return;   // a decoder sees the coded TUs of an inter CU only
        hevc_tu_t t{};
        t.x = (uint16_t)x;
        t.y = (uint16_t)y;
        t.log2_size = (uint8_t)log2;
        t.c_idx = (uint8_t)c;
        const int qpy = cu_qp(), bd_off = 6 * (p.bit_depth - 8);
        t.qp = (uint8_t)(c ? chroma_qp(qpy + (c == 1 ? cb_off : cr_off), bd_off) : qpy + bd_off);
        t.flags = (uint8_t)((inter ? 0 : HEVC_TU_INTRA) | (coded ? HEVC_TU_CODED : 0) |
                            (coded && cu_bypass ? HEVC_TU_BYPASS : 0));
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
        if ((cbf_luma || cb || cr) && p.qp_delta && !qp_delta_coded) cu_qp_delta();
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

    // The picture's slice segments in tile scan: [start, end) CtbAddrInTs and whether the
    // segment is dependent.  Cuts are drawn; with tiles a slice or segment either lies in one
    // tile or holds whole tiles, and under WPP a segment that starts inside a CTB row ends
    // in that row (7.4.7.1 constraints).
    struct Segment {
        int start, end;
        bool dependent;
    };
    std::vector<Segment> draw_segments() {
        const int n = wctb * hctb;
        std::vector<uint8_t> cut((size_t)n + 1, 0), indep((size_t)n + 1, 0);
        cut[0] = indep[0] = 1;
        cut[(size_t)n] = 1;
        const int max_seg = std::max(1, cfg.slices);
        const double p_cut = max_seg > 1 ? std::min(0.5, 1.5 * (max_seg - 1) / n) : 0.0;
        std::vector<uint8_t> tile_start((size_t)n + 1, 0), split_tile((size_t)p.tiles(), 0);
        for (int ts = 0; ts < n; ts++) tile_start[(size_t)ts] = ts == 0 || ctb_tile[(size_t)ts_to_rs[(size_t)ts]] != ctb_tile[(size_t)ts_to_rs[(size_t)ts - 1]];
        tile_start[(size_t)n] = 1;
        if (p.tiles() > 1) {
            for (int t = 0; t < p.tiles(); t++) split_tile[(size_t)t] = max_seg > 1 && u01() < 0.4;
            for (int ts = 1; ts < n; ts++) {
                const int t = ctb_tile[(size_t)ts_to_rs[(size_t)ts]];
                if (tile_start[(size_t)ts]) {
                    const int tp = ctb_tile[(size_t)ts_to_rs[(size_t)ts - 1]];
                    const bool forced = split_tile[(size_t)t] || split_tile[(size_t)tp];
                    cut[(size_t)ts] = forced || (max_seg > 1 && u01() < 0.5);
                    indep[(size_t)ts] = forced;
                } else if (split_tile[(size_t)t]) {
                    cut[(size_t)ts] = u01() < p_cut * 2;
                }
            }
        } else {
            for (int ts = 1; ts < n; ts++) cut[(size_t)ts] = u01() < p_cut;
            if (p.wpp) {   // a segment starting inside a row ends in it
                bool mid = false;
                for (int ts = 1; ts <= n; ts++) {
                    if (ts % wctb == 0 && mid) cut[(size_t)ts] = 1;
                    if (ts % wctb == 0) mid = false;
                    if (cut[(size_t)ts] && ts % wctb != 0) mid = true;
                }
            }
        }
        std::vector<Segment> segs;
        for (int ts = 0; ts < n;) {
            int e = ts + 1;
            while (!cut[(size_t)e]) e++;
            const bool dep = !indep[(size_t)ts] && p.dependent_slices && u01() < 0.5;
            segs.push_back({ts, e, dep});
            ts = e;
        }
        return segs;
    }

    // The reference list sizes and TMVP of a P/B picture: the same in every slice of it.
    struct InterPic {
        bool tmvp = false, col_l0 = true;
        int col_ref = 0;
        int total_curr = 0;                     // NumPicTotalCurr
        bool mod[2] = {false, false};           // ref_pic_list_modification_flag_lX
        std::vector<int> entry[2];              // list_entry_lX
    };
    // The lists (8.3.4): RefPicListTemp0 repeats StCurrBefore, StCurrAfter, LtCurr,
    // RefPicListTemp1 StCurrAfter, StCurrBefore, LtCurr; each list takes its first entries,
    // or with ref_pic_list_modification_flag_lX the entries list_entry_lX names.
    InterPic draw_inter(const PicPlan& pl, GopState& gop) {
        InterPic ip;
        std::vector<int> before, after, lt;
        for (size_t i = 0; i < pl.neg.size(); i++)
            if (pl.neg_used[i]) before.push_back(pl.neg[i]);
        for (size_t i = 0; i < pl.pos.size(); i++)
            if (pl.pos_used[i]) after.push_back(pl.pos[i]);
        for (size_t i = 0; i < pl.lt.size(); i++)
            if (pl.lt_used[i]) lt.push_back(pl.lt[i]);
        std::vector<int> src[2] = {before, after};
        src[0].insert(src[0].end(), after.begin(), after.end());
        src[1].insert(src[1].end(), before.begin(), before.end());
        for (auto& v : src) v.insert(v.end(), lt.begin(), lt.end());
        const bool override_refs = u01() < 0.7;
        num_ref[0] = override_refs ? uni(1, 4) : 1;
        num_ref[1] = slice_type == 0 ? (override_refs ? uni(1, 4) : 1) : 0;
        ip.total_curr = (int)src[0].size();
        for (int l = 0; l < (slice_type == 0 ? 2 : 1); l++)
            if (p.list_mod && ip.total_curr > 1 && u01() < 0.6) {
                ip.mod[l] = true;
                for (int i = 0; i < num_ref[l]; i++) ip.entry[l].push_back(uni(0, ip.total_curr - 1));
            }
        auto list_poc = [&](int l, int i) {
            return src[l][(size_t)(ip.mod[l] ? ip.entry[l][(size_t)i] : i % ip.total_curr)];
        };
        ip.tmvp = p.tmvp && u01() < 0.8;
        if (ip.tmvp) {
            ip.col_l0 = slice_type == 1 || u01() < 0.5;
            const int l = ip.col_l0 ? 0 : 1, nl = num_ref[l];
            std::vector<int> ok;   // entries decoded after the last picture without TMVP
            for (int i = 0; i < nl; i++) {
                const int poc = list_poc(l, i);
                if (gop.decode_idx_of_poc[(size_t)poc] >= gop.tmvp_barrier) ok.push_back(i);
            }
            if (ok.empty()) ip.tmvp = false;
            else ip.col_ref = ok[(size_t)uni(0, (int)ok.size() - 1)];
        }
        if (!ip.tmvp) gop.tmvp_barrier = pl.decode_idx;
        return ip;
    }

    // slice_segment_header() (7.3.6.1) up to (not including) the entry points; draws the
    // slice's values for an independent segment.  Returns the initType.
    int segment_header(Bits& b, const Segment& sg, int poc, const InterPic& ip) {
        const bool idr = plan->nal_type == 19 || plan->nal_type == 20;   // IDR_W_RADL, IDR_N_LP
        const bool irap = plan->nal_type >= 16 && plan->nal_type <= 23;
        const bool intra = slice_type == 2;
        const int nctb = wctb * hctb;
        b.bit(sg.start == 0);   // first_slice_segment_in_pic_flag
        if (irap) b.bit(plan->no_output_of_prior ? 1 : 0);   // no_output_of_prior_pics_flag
        b.ue((uint32_t)p.pps_id);   // slice_pic_parameter_set_id
        if (sg.start > 0) {
            if (p.dependent_slices) b.bit(sg.dependent ? 1 : 0);   // dependent_slice_segment_flag
            int bits = 0;
            while ((1 << bits) < nctb) bits++;
            b.put((uint32_t)ts_to_rs[(size_t)sg.start], bits);      // slice_segment_address
        }
        if (sg.dependent) return init_type;
        for (int i = 0; i < p.extra_bits; i++) b.bit(uni(0, 1));   // slice_reserved_flag
        b.ue((uint32_t)slice_type);
        if (p.output_flag) b.bit(plan->output ? 1 : 0);   // pic_output_flag
        if (!idr) {
            const uint32_t lsb_mask = (1u << p.poc_bits) - 1u;
            b.put((uint32_t)poc & lsb_mask, p.poc_bits);   // slice_pic_order_cnt_lsb
            const Rps t = rps_of(*plan);
            const int k = (int)p.rps_sets.size();
            int in_sps = -1;
            for (int i = 0; i < k && in_sps < 0; i++)
                if (p.rps_sets[(size_t)i] == t) in_sps = i;
            if (in_sps >= 0 && u01() < 0.8) {
                b.bit(1);                      // short_term_ref_pic_set_sps_flag
                int bits = 0;
                while ((1 << bits) < k) bits++;
                if (k > 1) b.put((uint32_t)in_sps, bits);   // short_term_ref_pic_set_idx
            } else {
                b.bit(0);                      // short_term_ref_pic_set_sps_flag
                st_ref_pic_set(b, t, k, p.rps_sets, true, rng);
            }
            if (p.long_term) {
                b.ue((uint32_t)plan->lt.size());             // num_long_term_pics
                for (size_t i = 0; i < plan->lt.size(); i++) {
                    // the MSB is sent whenever it differs from the current picture's (low
                    // delay: then another kept picture may share the LSBs)
                    const bool msb = plan->lt_msb[i] || (poc >> p.poc_bits) != (plan->lt[i] >> p.poc_bits);
                    b.put((uint32_t)plan->lt[i] & lsb_mask, p.poc_bits);   // poc_lsb_lt
                    b.bit(plan->lt_used[i]);                 // used_by_curr_pic_lt_flag
                    b.bit(msb ? 1 : 0);                      // delta_poc_msb_present_flag
                    if (msb) b.ue((uint32_t)((poc >> p.poc_bits) - (plan->lt[i] >> p.poc_bits)));   // delta_poc_msb_cycle_lt
                }
            }
            if (p.tmvp) b.bit(ip.tmvp ? 1 : 0);   // slice_temporal_mvp_enabled_flag
        }
        sao_luma = sao_chroma = false;
        if (p.sao) {
            sao_luma = u01() < 0.85;
            sao_chroma = u01() < 0.85;
            b.bit(sao_luma ? 1 : 0);           // slice_sao_luma_flag
            b.bit(sao_chroma ? 1 : 0);         // slice_sao_chroma_flag
        }
        init_type = 0;
        if (!intra) {
            const bool override_refs = num_ref[0] != 1 || (slice_type == 0 && num_ref[1] != 1) || u01() < 0.3;
            b.bit(override_refs ? 1 : 0);      // num_ref_idx_active_override_flag
            if (override_refs) {
                b.ue((uint32_t)(num_ref[0] - 1));
                if (slice_type == 0) b.ue((uint32_t)(num_ref[1] - 1));
            }
            if (p.list_mod && ip.total_curr > 1) {   // ref_pic_lists_modification() (7.3.6.2)
                int bits = 0;
                while ((1 << bits) < ip.total_curr) bits++;
                for (int l = 0; l < (slice_type == 0 ? 2 : 1); l++) {
                    b.bit(ip.mod[l] ? 1 : 0);   // ref_pic_list_modification_flag_lX
                    if (ip.mod[l])
                        for (int e : ip.entry[l]) b.put((uint32_t)e, bits);   // list_entry_lX
                }
            }
            mvd_l1_zero = false;
            if (slice_type == 0) {
                mvd_l1_zero = u01() < 0.3;
                b.bit(mvd_l1_zero ? 1 : 0);    // mvd_l1_zero_flag
            }
            const bool cabac_init = u01() < 0.3;
            b.bit(cabac_init ? 1 : 0);         // cabac_init_flag
            init_type = slice_type == 1 ? (cabac_init ? 2 : 1) : (cabac_init ? 1 : 2);
            if (ip.tmvp) {
                if (slice_type == 0) b.bit(ip.col_l0 ? 1 : 0);                  // collocated_from_l0_flag
                if (num_ref[ip.col_l0 ? 0 : 1] > 1) b.ue((uint32_t)ip.col_ref);  // collocated_ref_idx
            }
            if (p.wp) pred_weight_table(b);
            max_merge = cfg.max_merge ? cfg.max_merge : uni(1, 5);
            b.ue((uint32_t)(5 - max_merge));   // five_minus_max_num_merge_cand
        }
        qp = uni(cfg.qp_min, cfg.qp_max);
        b.se(qp - 26);                         // slice_qp_delta
        cb_off = p.cb_qp_offset;
        cr_off = p.cr_qp_offset;
        if (p.slice_chroma_offsets) {
            const int scb = uni(std::max(-12, -12 - p.cb_qp_offset), std::min(12, 12 - p.cb_qp_offset));
            const int scr = uni(std::max(-12, -12 - p.cr_qp_offset), std::min(12, 12 - p.cr_qp_offset));
            b.se(scb);                         // slice_cb_qp_offset
            b.se(scr);                         // slice_cr_qp_offset
            cb_off += scb;
            cr_off += scr;
        }
        bool dbk_disabled = p.dbk_disabled;
        if (p.dbk_override) {
            const bool ov = u01() < 0.5;
            b.bit(ov ? 1 : 0);                 // deblocking_filter_override_flag
            if (ov) {
                dbk_disabled = u01() < 0.3;
                b.bit(dbk_disabled ? 1 : 0);   // slice_deblocking_filter_disabled_flag
                if (!dbk_disabled) {
                    b.se(uni(-6, 6));          // slice_beta_offset_div2
                    b.se(uni(-6, 6));          // slice_tc_offset_div2
                }
            }
        }
        if (p.lf_across_slices && (sao_luma || sao_chroma || !dbk_disabled))
            b.bit(u01() < 0.5 ? 1 : 0);        // slice_loop_filter_across_slices_enabled_flag
        return init_type;
    }
    int init_type = 0;

    // slice_segment_data() (7.3.8.1) of one segment into d: CTUs in tile scan, each
    // followed by end_of_slice_segment_flag, and end_of_subset_one_bit + byte_alignment()
    // before a new tile or (WPP) a new CTB row; starts[k] is the byte offset of substream k.
    // Contexts (9.3.1): initialised at the segment (unless dependent), at each tile, and
    // at each row under WPP, where they come from the state stored after the second CTB of
    // the row above when that CTB is available.
    void segment_data(Bits& d, const Segment& sg, std::vector<size_t>& starts) {
        Contexts wpp_saved;
        for (int ts = sg.start; ts < sg.end; ts++) {
            const int rs = ts_to_rs[(size_t)ts], rx = rs % wctb, ry = rs / wctb;
            cur_tile = ctb_tile[(size_t)rs];
            cur_slice = ctb_slice[(size_t)rs];
            const bool new_tile = ts == 0 || ctb_tile[(size_t)ts_to_rs[(size_t)ts - 1]] != cur_tile;
            const bool row_start = p.wpp && rx == 0;
            if (ts == sg.start || new_tile || row_start) {
                starts.push_back(d.buf.size());
                E.start(&d);
                const bool quirk_tiles = cfg.ref_quirks & HEVCGEN_QUIRK_TILES_PCM;
                if (new_tile && !(quirk_tiles && (ts != sg.start || sg.dependent))) {
                    C.init(init_type, qp);
                } else if (new_tile) {
                } else if (row_start) {
                    if (avail((rx + 1) << p.log2_ctb, (ry - 1) << p.log2_ctb)) C = wpp_saved;
                    else C.init(init_type, qp);
                } else if (!sg.dependent) {
                    C.init(init_type, qp);
                }
                if (new_tile || row_start || !sg.dependent || (cfg.ref_quirks & HEVCGEN_QUIRK_DEPENDENT)) {
                    first_qg = true;
                    last_cu_qp = qp;   // qPY_PREV of the group; also the QpY a PCM CU takes in quirk mode
                }
            }
            if (p.sao && (sao_luma || sao_chroma)) sao(rx, ry);
            coding_quadtree(rx << p.log2_ctb, ry << p.log2_ctb, p.log2_ctb, 0);
            if (p.wpp && rx == 1) wpp_saved = C;
            const bool last = ts == sg.end - 1;
            E.terminate(last);   // end_of_slice_segment_flag
            if (last) {
                d.align_zero();  // the flush's last bit is rbsp_stop_one_bit
            } else {
                const int nrs = ts_to_rs[(size_t)ts + 1];
                if (ctb_tile[(size_t)nrs] != cur_tile || (p.wpp && nrs % wctb == 0)) {
                    E.terminate(1);   // end_of_subset_one_bit; the flush ends in alignment_bit_equal_to_one
                    if ((cfg.ref_quirks & HEVCGEN_QUIRK_TILES_PCM) && p.tiles() > 1 && d.n == 0) d.put(0x80, 8);
                    d.align_zero();
                }
            }
        }
    }

    // Every slice segment NAL unit of the picture into out.
    const PicPlan* plan = nullptr;
    void code_picture(const PicPlan& pl, GopState& gop, std::vector<uint8_t>& out, bool aud,
                      const std::vector<uint8_t>& param_sets) {
        plan = &pl;
        if (p.extra && aud) nal(out, 35, access_unit_delimiter(), pl.tid);
        out.insert(out.end(), param_sets.begin(), param_sets.end());   // a new SPS and PPS (after the AUD)
        if (p.extra)
            for (int i = uni(0, 2); i > 0; i--) nal(out, 39, sei_user_data(), pl.tid);   // PREFIX_SEI
        const int poc = pl.poc;
        slice_type = pl.slice_type;
        const bool intra = slice_type == 2;
        const int nal_type = pl.nal_type;
        InterPic ip;
        if (!intra) ip = draw_inter(pl, gop);
        else gop.tmvp_barrier = pl.decode_idx;   // slice_temporal_mvp_enabled_flag 0 (or absent, IDR)
        const std::vector<Segment> segs = draw_segments();
        int slice_addr = 0;
        for (const Segment& sg : segs) {
            if (!sg.dependent || (cfg.ref_quirks & HEVCGEN_QUIRK_DEPENDENT)) slice_addr = ts_to_rs[(size_t)sg.start];
            for (int ts = sg.start; ts < sg.end; ts++) ctb_slice[(size_t)ts_to_rs[(size_t)ts]] = slice_addr;
        }
        for (const Segment& sg : segs) {
            Bits h;
            segment_header(h, sg, poc, ip);
            Bits d;
            std::vector<size_t> starts;
            segment_data(d, sg, starts);
            const bool entry = p.tiles() > 1 || p.wpp;
            std::vector<uint32_t> sizes;   // substream sizes in NAL bytes (emulation prevention included)
            for (size_t k = 0; k + 1 < starts.size(); k++) sizes.push_back((uint32_t)(starts[k + 1] - starts[k]));
            const bool quirk_dep = sg.dependent && (cfg.ref_quirks & HEVCGEN_QUIRK_DEPENDENT);
            std::vector<uint8_t> ext;   // slice_segment_header_extension_data_byte
            if (p.extra)
                for (int i = uni(0, 3); i > 0; i--) ext.push_back((uint8_t)uni(0, 255));
            for (int iter = 0;; iter++) {
                Bits hh = h;
                if (quirk_dep) {
                    if (hh.n) hh.trailing();
                    std::vector<uint8_t> rbsp = hh.buf;
                    rbsp.insert(rbsp.end(), d.buf.begin(), d.buf.end());
                    nal(out, nal_type, rbsp, pl.tid);
                    break;
                }
                if (entry) {
                    hh.ue((uint32_t)sizes.size());   // num_entry_point_offsets
                    if (!sizes.empty()) {
                        uint32_t mx = 1;
                        for (uint32_t v : sizes) mx = std::max(mx, v);
                        int len = 1;
                        while (len < 32 && ((mx - 1) >> len) != 0) len++;
                        hh.ue((uint32_t)(len - 1));  // offset_len_minus1
                        for (uint32_t v : sizes) hh.put(v - 1, len);   // entry_point_offset_minus1
                    }
                }
                if (p.extra) {
                    hh.ue((uint32_t)ext.size());   // slice_segment_header_extension_length
                    for (uint8_t v : ext) hh.put(v, 8);
                }
                hh.trailing();   // byte_alignment()
                std::vector<uint8_t> rbsp = hh.buf;
                const size_t hsize = rbsp.size();
                rbsp.insert(rbsp.end(), d.buf.begin(), d.buf.end());
                const std::vector<size_t> pos = nal_positions(rbsp);
                std::vector<uint32_t> got;
                for (size_t k = 0; k + 1 < starts.size(); k++)
                    got.push_back((uint32_t)(pos[hsize + starts[k + 1]] - pos[hsize + starts[k]]));
                if (got == sizes || iter == 8) {
                    nal(out, nal_type, rbsp, pl.tid);
                    break;
                }
                sizes = got;
            }
        }
        if (p.extra) {
            for (int i = uni(0, 1); i > 0; i--) nal(out, 40, sei_user_data(), pl.tid);   // SUFFIX_SEI
            if (uni(0, 2) == 0) nal(out, 38, filler_data(), pl.tid);                     // FD_NUT
        }
    }

    // access_unit_delimiter_rbsp() (7.3.2.5): pic_type 2 (I, P and B slices may follow)
    static std::vector<uint8_t> access_unit_delimiter() {
        Bits b;
        b.put(2, 3);
        b.trailing();
        return b.buf;
    }

    // sei_rbsp() (7.3.2.4) with one user_data_unregistered message (D.2.7): payloadType 5,
    // a 16-byte UUID and some random bytes; a decoder ignores it
    std::vector<uint8_t> sei_user_data() {
        Bits b;
        const int size = 16 + uni(0, 300);
        b.put(5, 8);   // last_payload_type_byte
        for (int v = size; ; v -= 255) {   // ff_byte ... last_payload_size_byte
            if (v >= 255) {
                b.put(255, 8);
            } else {
                b.put((uint32_t)v, 8);
                break;
            }
        }
        for (int i = 0; i < size; i++) b.put((uint32_t)uni(0, 255), 8);
        b.trailing();
        return b.buf;
    }

    // filler_data_rbsp() (7.3.2.8): 0xFF bytes
    std::vector<uint8_t> filler_data() {
        Bits b;
        for (int i = uni(1, 64); i > 0; i--) b.put(0xFF, 8);
        b.trailing();
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
    // sign data hiding (7.3.8.11, 7.4.9.11): in a sub-block whose first and last nonzero
    // scan positions are more than 3 apart, the sign of the first is not coded but is the
    // parity of the sub-block's sum of magnitudes (odd: negative); the drawn sign obeys it
    const bool sdh = p.sdh && !cu_bypass;
    if (sdh)
        for (int i = 0; i <= (last >> 4); i++) {
            int lo = -1, hi = -1, sum = 0;
            for (int q = 0; q < 16 && 16 * i + q <= last; q++) {
                const auto xy = at(16 * i + q);
                const int v = lv[xy.second * n + xy.first];
                if (!v) continue;
                if (lo < 0) lo = q;
                hi = q;
                sum += std::abs(v);
            }
            if (lo < 0 || hi - lo <= 3) continue;
            const auto xy = at(16 * i + lo);
            int16_t& v = lv[xy.second * n + xy.first];
            v = (int16_t)((sum & 1) ? -std::abs(v) : std::abs(v));
        }
    // transform_skip_flag: first syntax element of a 4x4 block's residual_coding()
    if (p.tskip && !cu_bypass && log2 == 2) {
        const bool ts = u01() < cfg.p_tskip;
        E.decision(C.tskip[c ? 1 : 0], ts);
        if (ts) tus.back().flags |= HEVC_TU_TSKIP;
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
        int lo_q = -1, hi_q = -1;   // firstSigScanPos, lastSigScanPos in the sub-block
        if (i == last_sb) {
            sig.push_back(lv[lxy.second * n + lxy.first]);
            lo_q = hi_q = last & 15;
        }
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
            if (v) {
                sig.push_back(v);
                if (hi_q < 0) hi_q = q;
                lo_q = q;
            }
        }
        if (sig.empty()) continue;
        const bool hidden = sdh && hi_q - lo_q > 3;
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
        for (int k = 0; k < ns; k++)
            if (!(hidden && k == ns - 1)) E.bypass(sig[(size_t)k] < 0);
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
// Merge candidates: the left / above CTB when in the slice (raster address at or after
// SliceAddrRs) and the tile; components the slice's SAO flags leave off have no syntax.
void Picture::sao(int rx, int ry) {
    const int rs = ry * wctb + rx;
    bool merge = false;
    if (rx > 0 && rs > cur_slice && ctb_tile[(size_t)rs] == ctb_tile[(size_t)rs - 1]) {
        merge = u01() < 0.3;
        E.decision(C.sao_merge, merge);
    }
    if (!merge && ry > 0 && rs - wctb >= cur_slice && ctb_tile[(size_t)rs] == ctb_tile[(size_t)(rs - wctb)]) {
        merge = u01() < 0.3;
        E.decision(C.sao_merge, merge);
    }
    if (merge) return;
    int type = 0;
    for (int c = 0; c < 3; c++) {
        if (c == 0 ? !sao_luma : !sao_chroma) continue;
        if (c < 2) {   // sao_type_idx: TR cMax 2, first bin context-coded
            type = uni(0, 2);
            E.decision(C.sao_type, type != 0);
            if (type) E.bypass(type == 2);
        }
        if (!type) continue;
        int abs_v[4];
        // sao_offset_abs: TR cMax (1 << (Min(BitDepth, 10) - 5)) - 1, bypass (7.4.9.3.2)
        const int sao_max = (1 << (std::min(p.bit_depth, 10) - 5)) - 1;
        for (int k = 0; k < 4; k++) {
            abs_v[k] = uni(0, sao_max);
            for (int b = 0; b < abs_v[k]; b++) E.bypass(1);
            if (abs_v[k] < sao_max) E.bypass(0);
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

namespace {

// The coded sequence (pictures in decode order), in IDR periods of idr_period pictures (the
// whole stream when 0); POCs restart at 0 in each.  Low delay: POC = decode index within the
// period, each P/B picture using some of the last max_refs pictures.  Random access
// (ra_gop = G > 1): after the IDR picture, mini-GOPs of G pictures: the last one first
// (predicted from earlier pictures), then the ones between by bisection, each predicted
// from the two pictures around it (and one earlier one when max_refs allows).  A picture's
// RPS keeps every earlier-decoded picture of its period that it or a later picture uses
// (8.3.2).  An IDR picture after the first draws no_output_of_prior_pics_flag; with
// p_no_output a picture draws pic_output_flag = 0.
std::vector<PicPlan> plan_sequence(const hevcgen_cfg_t& cfg, std::mt19937_64& rng) {
    auto u01 = [&]() { return std::uniform_real_distribution<double>(0.0, 1.0)(rng); };
    std::vector<PicPlan> plan;
    const int period = !cfg.inter ? 1 : cfg.idr_period > 0 ? cfg.idr_period : cfg.pictures;
    for (int first = 0; first < cfg.pictures; first += period) {
        const int n = std::min(period, cfg.pictures - first);
        std::vector<int> order{0};
        std::vector<std::vector<int>> refs;   // POCs each picture uses
        // random access with cra: some mini-GOPs end in a CRA picture (intra, POCs go on);
        // their inner pictures are its leading pictures: RADL from POC radl_from on (they
        // use only the CRA picture and other RADL pictures), RASL below it
        std::vector<int> cra, radl_from;
        std::map<int, int> tid_of;   // TemporalId: the bisection depth (with temporal)
        if (cfg.inter) {
            const int g = std::max(1, cfg.ra_gop);
            std::function<void(int, int, int)> bisect = [&](int lo, int hi, int depth) {
                if (hi - lo < 2) return;
                const int mid = (lo + hi) / 2;
                order.push_back(mid);
                tid_of[mid] = cfg.temporal ? std::min(6, depth) : 0;
                bisect(lo, mid, depth + 1);
                bisect(mid, hi, depth + 1);
            };
            for (int base = 0; base < n - 1; base += g) {
                const int anchor = std::min(base + g, n - 1);
                order.push_back(anchor);
                if (cfg.cra && g > 1 && u01() < 0.5) {   // a CRA picture, its mini-GOP's inner pictures leading
                    cra.push_back(anchor);
                    radl_from.push_back(anchor - base >= 2 && u01() < 0.5 ? (base + anchor) / 2 : anchor);
                }
                bisect(base, anchor, 1);
            }
        }
        // long-term (low delay only): from the period's third picture on, its IDR picture
        // (POC 0) is a long-term reference picture, kept in every RPS, used or not
        const bool lt_mode = cfg.long_term && cfg.inter && cfg.ra_gop < 2;
        std::vector<int> lt_used(order.size(), 0);
        for (size_t j = 0; j < order.size(); j++) {
            const int poc = order[j];
            std::vector<int> r;
            if (j > 0) {
                if (cfg.ra_gop < 2) {   // low delay: the last max_refs pictures, at least one used
                    const int lowest = lt_mode && j >= 2 ? 1 : 0;
                    for (int q = poc - 1; q >= lowest && q >= poc - cfg.max_refs; q--)
                        if (u01() < 0.7 || r.empty()) r.push_back(q);
                    if (lt_mode && j >= 2) lt_used[j] = u01() < 0.5;
                } else if (std::find(cra.begin(), cra.end(), poc) == cra.end()) {
                    // the IRAP picture this one follows in decode order: its trailing pictures
                    // use only pictures from it on; its RADL pictures only it and RADL pictures
                    int floor = 0;
                    for (size_t i = 0; i < j; i++)
                        if (std::find(cra.begin(), cra.end(), order[i]) != cra.end()) {
                            const size_t c = (size_t)(std::find(cra.begin(), cra.end(), order[i]) - cra.begin());
                            if (poc > order[i]) floor = order[i];
                            else if (poc >= radl_from[c]) floor = radl_from[c] == poc ? order[i] : radl_from[c];
                        }
                    std::vector<int> past, future;   // decoded before: below and above in output order
                    for (size_t i = 0; i < j; i++) {
                        if (order[i] < floor && !(floor > poc)) continue;
                        (order[i] < poc ? past : future).push_back(order[i]);
                    }
                    std::sort(past.begin(), past.end(), std::greater<int>());
                    std::sort(future.begin(), future.end());
                    if (!past.empty() && !(floor > poc)) r.push_back(past[0]);
                    if (!future.empty()) r.push_back(future[0]);
                    if (!(floor > poc) && (int)r.size() < cfg.max_refs && past.size() > 1 &&
                        tid_of[past[1]] <= tid_of[poc] && u01() < 0.5)
                        r.push_back(past[1]);   // a picture of a higher sub-layer is never a reference
                }
            }
            refs.push_back(r);
        }
        for (size_t j = 0; j < order.size(); j++) {
            PicPlan pl;
            pl.poc = order[j];
            pl.decode_idx = (int)plan.size();
            pl.tid = tid_of.count(pl.poc) ? tid_of[pl.poc] : 0;
            const bool is_cra = std::find(cra.begin(), cra.end(), pl.poc) != cra.end();
            pl.slice_type = j == 0 || is_cra ? 2 : (u01() < cfg.p_b ? 0 : 1);
            pl.output = !(cfg.p_no_output > 0 && u01() < cfg.p_no_output);
            pl.no_output_of_prior = j == 0 && first > 0 && u01() < 0.3;
            pl.nal_type = j == 0 ? (u01() < 0.5 ? 19 : 20) : is_cra ? 21 : 1;   // IDR_W_RADL / IDR_N_LP, CRA_NUT, TRAIL_R
            for (size_t c = 0; c < cra.size(); c++)   // a leading picture: RASL_R or RADL_R
                if (j > 0 && pl.poc < cra[c] && pl.poc > cra[c] - std::max(1, cfg.ra_gop) &&
                    std::find(order.begin(), order.begin() + (long)j, cra[c]) != order.begin() + (long)j)
                    pl.nal_type = pl.poc >= radl_from[c] ? 7 : 9;
            if (cfg.temporal && j > 0 && pl.nal_type == 1 && pl.tid > 0 && u01() < 0.6) {
                // a sub-layer switching point where the plan allows one (7.4.2.2): TSA when
                // neither it nor a later picture of its sub-layer or above uses a picture of
                // those sub-layers decoded before it; else STSA, the same within its sub-layer
                std::map<int, size_t> at;   // POC -> decode position in the period
                for (size_t i = 0; i < order.size(); i++) at[order[i]] = i;
                auto allowed = [&](bool tsa) {
                    auto hit = [&](int r, int t) { return tsa ? tid_of[r] >= t : tid_of[r] == t; };
                    for (int r : refs[j])
                        if (hit(r, pl.tid)) return false;
                    for (size_t m = j + 1; m < order.size(); m++) {
                        const int tm = tid_of[order[m]];
                        if (tsa ? tm < pl.tid : tm != pl.tid) continue;
                        for (int r : refs[m])
                            if (at[r] < j && hit(r, pl.tid)) return false;
                    }
                    return true;
                };
                if (allowed(true)) pl.nal_type = 3;          // TSA_R
                else if (allowed(false)) pl.nal_type = 5;    // STSA_R
            }
            if (cfg.nonref_types && j > 0 &&
                (pl.nal_type == 1 || pl.nal_type == 3 || pl.nal_type == 5 || pl.nal_type == 7 || pl.nal_type == 9)) {
                // a picture no later one uses: the sub-layer non-reference type (TRAIL_N,
                // TSA_N, STSA_N, RADL_N, RASL_N), which 8.3.1 leaves out of prevTid0Pic
                bool used = false;
                for (size_t m = j + 1; m < order.size() && !used; m++)
                    used = std::find(refs[m].begin(), refs[m].end(), pl.poc) != refs[m].end();
                if (!used) pl.nal_type -= 1;
            }
            if (j > 0) {
                std::vector<int> keep;   // decoded before j, used by j or by a later picture
                for (size_t i = 0; i < j; i++) {
                    bool needed = false;
                    for (size_t m = j; m < order.size() && !needed; m++)
                        needed = std::find(refs[m].begin(), refs[m].end(), order[i]) != refs[m].end();
                    if (needed) keep.push_back(order[i]);
                }
                if (lt_mode && j == 1 && std::find(keep.begin(), keep.end(), 0) == keep.end())
                    keep.push_back(0);   // kept for the pictures that take it as long-term
                if (lt_mode && j >= 2) {
                    keep.erase(std::remove(keep.begin(), keep.end(), 0), keep.end());
                    pl.lt.push_back(0);
                    pl.lt_used.push_back(lt_used[j]);
                    pl.lt_msb.push_back(u01() < 0.3);
                }
                std::sort(keep.begin(), keep.end());
                for (auto it = keep.rbegin(); it != keep.rend(); ++it)
                    if (*it < pl.poc) pl.neg.push_back(*it);
                for (int q : keep)
                    if (q > pl.poc) pl.pos.push_back(q);
                auto used = [&](int q) { return (int)(std::find(refs[j].begin(), refs[j].end(), q) != refs[j].end()); };
                for (int q : pl.neg) pl.neg_used.push_back(used(q));
                for (int q : pl.pos) pl.pos_used.push_back(used(q));
            }
            plan.push_back(pl);
        }
    }
    return plan;
}

// sps_max_num_reorder_pics: the most pictures that precede one in decode order and follow it
// in output order; sps_max_dec_pic_buffering_minus1: room for the largest RPS, the pictures
// waiting for output and the current one.
void dpb_sizes(const std::vector<PicPlan>& plan, int& num_reorder, int& dpb_minus1) {
    num_reorder = 0;
    size_t rps = 0, start = 0;   // start: the IDR picture of j's period (output order restarts there)
    for (size_t j = 0; j < plan.size(); j++) {
        if (plan[j].nal_type == 19 || plan[j].nal_type == 20) start = j;
        int c = 0;
        for (size_t i = start; i < j; i++) c += plan[i].poc > plan[j].poc;
        num_reorder = std::max(num_reorder, c);
        rps = std::max(rps, plan[j].neg.size() + plan[j].pos.size() + plan[j].lt.size());
    }
    dpb_minus1 = std::min(15, std::max(1, (int)rps + num_reorder));
}

}  // namespace

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
    cfg->slices = 1;
    cfg->tile_cols = 1;
    cfg->tile_rows = 1;
}

hevcgen_stream_t* hevcgen_stream(const hevcgen_cfg_t* cfg) {
    if (!cfg || cfg->width <= 0 || cfg->height <= 0 || (cfg->width & 7) || (cfg->height & 7) || cfg->pictures < 1 ||
        cfg->log2_ctb < 4 || cfg->log2_ctb > 6 || cfg->max_level < 1 || cfg->qp_min < 0 || cfg->qp_max > 51 ||
        cfg->qp_min > cfg->qp_max || cfg->max_refs < 1 || cfg->max_refs > 4 || cfg->max_mvd < 1 ||
        cfg->max_mvd > 1 << 14 || cfg->max_merge < 0 || cfg->max_merge > 5 || cfg->depth_inter < 0 ||
        cfg->depth_inter > 2 || cfg->slices < 1 || cfg->tile_cols < 1 || cfg->tile_rows < 1 || cfg->scaling < 0 ||
        cfg->scaling > 3 || cfg->qp_delta_depth < 0 ||
        (cfg->wpp && cfg->dependent_slices && (cfg->ref_quirks & HEVCGEN_QUIRK_DEPENDENT)) || cfg->idr_period < 0 ||
        (cfg->bit_depth != 0 && cfg->bit_depth != 8 && cfg->bit_depth != 10))
        return nullptr;
    std::mt19937_64 rng(cfg->seed);
    auto uni = [&](int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); };
    auto coin = [&]() { return uni(0, 1) == 1; };
    Params p{cfg->width, cfg->height, cfg->log2_ctb, cfg->sao ? 1 : 0};
    const int ctb = 1 << p.log2_ctb;
    // what depends on the picture size (it changes at an IDR picture with resize): the
    // tiles (as many as Main's minimum tile size of 256 x 64 luma samples allows), the
    // cropping window and the tile scan
    int wctb = 0, hctb = 0;
    std::vector<int> ts_to_rs, ctb_tile;
    auto layout = [&](int W, int H) {
        p.W = W;
        p.H = H;
        wctb = (W + ctb - 1) / ctb;
        hctb = (H + ctb - 1) / ctb;
        {
            const int min_w = (256 + ctb - 1) / ctb, min_h = (64 + ctb - 1) / ctb;
            const int nc = p.wpp ? 1 : std::max(1, std::min(cfg->tile_cols, wctb / min_w));
            const int nr = p.wpp ? 1 : std::max(1, std::min(cfg->tile_rows, hctb / min_h));
            p.uniform_tiles = coin() ? 1 : 0;
            auto bounds = [&](int n, int total, int min_size, std::vector<int>& bd) {
                bd.assign(1, 0);
                if (p.uniform_tiles) {
                    for (int i = 1; i <= n; i++) bd.push_back((i * total) / n);
                    return;
                }
                int left = total;
                for (int i = 0; i < n - 1; i++) {
                    const int sz = uni(min_size, left - min_size * (n - 1 - i));
                    bd.push_back(bd.back() + sz);
                    left -= sz;
                }
                bd.push_back(total);
            };
            bounds(nc, wctb, min_w, p.col_bd);
            bounds(nr, hctb, min_h, p.row_bd);
            p.lf_across_tiles = coin() ? 1 : 0;
        }
        if (cfg->crop) {   // the window keeps at least 16 x 16 luma samples
            const int mx = std::min(8, (p.W - 16) / 8), my = std::min(8, (p.H - 16) / 8);
            p.crop[0] = uni(0, std::max(0, mx));
            p.crop[1] = uni(0, std::max(0, mx));
            p.crop[2] = uni(0, std::max(0, my));
            p.crop[3] = uni(0, std::max(0, my));
        }
        // tile scan (6.5.1): CtbAddrTsToRs and the TileId of each raster address
        ts_to_rs.clear();
        ctb_tile.assign((size_t)wctb * hctb, 0);
        for (size_t j = 0; j + 1 < p.row_bd.size(); j++)
            for (size_t i = 0; i + 1 < p.col_bd.size(); i++)
                for (int y = p.row_bd[j]; y < p.row_bd[j + 1]; y++)
                    for (int x = p.col_bd[i]; x < p.col_bd[i + 1]; x++) {
                        ts_to_rs.push_back(y * wctb + x);
                        ctb_tile[(size_t)y * wctb + x] = (int)(j * (p.col_bd.size() - 1) + i);
                    }
    };
    if (cfg->inter) {
        p.inter = 1;
        p.dpb_minus1 = cfg->max_refs;
        p.amp = cfg->amp ? 1 : 0;
        p.tmvp = cfg->tmvp ? 1 : 0;
        p.wp = cfg->wp ? 1 : 0;
        p.log2_pml = uni(2, p.log2_ctb);
    }
    p.depth_inter = cfg->depth_inter;
    if (cfg->ra_gop > 1 && !cfg->inter) return nullptr;
    if (cfg->qp_delta_depth > 0) {
        p.qp_delta = 1;
        p.qp_delta_depth = std::min(cfg->qp_delta_depth - 1, p.log2_ctb - 3);
    }
    if (cfg->chroma_qp_offsets) {
        p.cb_qp_offset = uni(-12, 12);
        p.cr_qp_offset = uni(-12, 12);
        p.slice_chroma_offsets = coin() ? 1 : 0;
    }
    if (cfg->deblock_ctl) {
        p.dbk_ctl = 1;
        p.dbk_override = coin() ? 1 : 0;
        p.dbk_disabled = uni(0, 3) == 0 ? 1 : 0;
        p.beta_div2 = uni(-6, 6);
        p.tc_div2 = uni(-6, 6);
    }
    layout(cfg->width, cfg->height);
    p.wpp = cfg->wpp && p.tiles() == 1 ? 1 : 0;
    p.dependent_slices = cfg->dependent_slices ? 1 : 0;
    p.lf_across_slices = cfg->slices > 1 ? (coin() ? 1 : 0) : 1;
    p.bypass = cfg->p_bypass > 0 ? 1 : 0;
    p.tskip = cfg->p_tskip > 0 ? 1 : 0;
    p.sdh = cfg->sdh ? 1 : 0;
    p.bit_depth = cfg->bit_depth == 10 ? 10 : 8;
    if (cfg->p_pcm > 0) {
        p.pcm = 1;
        p.pcm_bits_y = uni(1, p.bit_depth);
        p.pcm_bits_c = uni(1, p.bit_depth);
        p.pcm_log2_min = uni(3, std::min(5, p.log2_ctb));
        p.pcm_log2_max = uni(p.pcm_log2_min, std::min(5, p.log2_ctb));
        p.pcm_lf_disabled = coin() ? 1 : 0;
    }
    p.scaling = cfg->scaling;
    p.output_flag = cfg->p_no_output > 0 ? 1 : 0;
    p.long_term = cfg->long_term ? 1 : 0;
    p.list_mod = cfg->list_mod ? 1 : 0;
    {   // POC LSBs: at least enough that every step from prevTid0Pic stays below half the range
        int need = 4;
        while ((1 << need) <= 2 * std::max(1, cfg->ra_gop) + 2) need++;
        p.poc_bits = cfg->poc_lsb_bits ? std::max(need, std::min(16, cfg->poc_lsb_bits)) : 8;
    }
    const std::vector<PicPlan> plan = plan_sequence(*cfg, rng);
    for (const PicPlan& pl : plan) p.max_tid = std::max(p.max_tid, pl.tid);
    if (cfg->inter) dpb_sizes(plan, p.num_reorder, p.dpb_minus1);
    if (cfg->inter && cfg->sps_rps) {   // the SPS holds the RPSs of most P/B pictures (the more frequent first)
        std::vector<std::pair<int, Rps>> count;
        for (const PicPlan& pl : plan) {
            if (pl.slice_type == 2) continue;
            const Rps r = rps_of(pl);
            auto it = std::find_if(count.begin(), count.end(), [&](const std::pair<int, Rps>& c) { return c.second == r; });
            if (it == count.end()) count.push_back({1, r});
            else it->first++;
        }
        std::stable_sort(count.begin(), count.end(),
                         [](const std::pair<int, Rps>& a, const std::pair<int, Rps>& b) { return a.first > b.first; });
        const size_t k = std::min<size_t>(count.size(), (size_t)uni(1, 8));
        for (size_t i = 0; i < k; i++) p.rps_sets.push_back(count[i].second);
    }
    p.extra = cfg->extra_syntax ? 1 : 0;
    if (p.extra) p.extra_bits = uni(0, 2);
    std::vector<uint8_t> out;
    if (p.extra) nal(out, 35, Picture::access_unit_delimiter());
    nal(out, 32, vps(p));
    nal(out, 33, sps(p, rng));
    // PPS variants (pps_count): the tools the configuration enables, each switched on or off
    // and drawn again per PPS; each picture refers to one of them
    std::vector<Params> ppss(1, p);
    auto vary = [&](Params& q) {
        q.qp_delta = p.qp_delta && coin() ? 1 : 0;
        if (q.qp_delta) q.qp_delta_depth = uni(0, p.log2_ctb - 3);
        if (cfg->chroma_qp_offsets) {
            q.cb_qp_offset = uni(-12, 12);
            q.cr_qp_offset = uni(-12, 12);
            q.slice_chroma_offsets = coin() ? 1 : 0;
        }
        if (cfg->deblock_ctl) {
            q.dbk_override = coin() ? 1 : 0;
            q.dbk_disabled = uni(0, 3) == 0 ? 1 : 0;
            q.beta_div2 = uni(-6, 6);
            q.tc_div2 = uni(-6, 6);
        }
        q.bypass = p.bypass && coin() ? 1 : 0;
        q.tskip = p.tskip && coin() ? 1 : 0;
        q.sdh = p.sdh && coin() ? 1 : 0;
        q.wp = p.wp && coin() ? 1 : 0;
        q.list_mod = p.list_mod && coin() ? 1 : 0;
        if (cfg->inter) q.log2_pml = uni(2, p.log2_ctb);
    };
    for (int i = 1; i < std::min(64, std::max(1, cfg->pps_count)); i++) {
        Params q = p;
        q.pps_id = i;
        vary(q);
        ppss.push_back(q);
    }
    for (const Params& q : ppss) nal(out, 34, pps(q, rng));
    auto* s = static_cast<hevcgen_stream_t*>(std::calloc(1, sizeof(hevcgen_stream_t)));
    s->pictures = cfg->pictures;
    s->num_tus = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->tus = static_cast<hevc_tu_t**>(std::calloc((size_t)cfg->pictures, sizeof(hevc_tu_t*)));
    s->num_coeffs = static_cast<uint64_t*>(std::calloc((size_t)cfg->pictures, sizeof(uint64_t)));
    s->coeffs = static_cast<int16_t**>(std::calloc((size_t)cfg->pictures, sizeof(int16_t*)));
    s->slice_type = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->num_pus = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->pus = static_cast<hevc_pu_t**>(std::calloc((size_t)cfg->pictures, sizeof(hevc_pu_t*)));
    s->poc = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->output = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    s->tid = static_cast<int32_t*>(std::calloc((size_t)cfg->pictures, sizeof(int32_t)));
    for (int k = 0; k < 4; k++) s->crop[k] = p.crop[k];
    GopState gop;
    gop.decode_idx_of_poc.assign((size_t)cfg->pictures, 0);
    for (int k = 0; k < cfg->pictures; k++) {
        const PicPlan& pl = plan[(size_t)k];
        std::vector<uint8_t> param_sets;
        if (cfg->resize && k > 0 && (pl.nal_type == 19 || pl.nal_type == 20) && coin()) {
            // a new size (multiples of 8, at least 16 x 16) from this IDR picture on: the SPS
            // and PPS are sent again before it (same ids; the new SPS is activated there)
            layout(std::max(16, cfg->width - 8 * uni(0, (cfg->width - 16) / 16)),
                   std::max(16, cfg->height - 8 * uni(0, (cfg->height - 16) / 16)));
            nal(param_sets, 33, sps(p, rng));
            for (Params& q : ppss) {   // the new size in every PPS variant
                q.W = p.W;
                q.H = p.H;
                q.col_bd = p.col_bd;
                q.row_bd = p.row_bd;
                q.uniform_tiles = p.uniform_tiles;
                q.lf_across_tiles = p.lf_across_tiles;
                for (int c = 0; c < 4; c++) q.crop[c] = p.crop[c];
                nal(param_sets, 34, pps(q, rng));
            }
        }
        Picture pic(*cfg, rng, ppss[ppss.size() > 1 ? (size_t)uni(0, (int)ppss.size() - 1) : 0]);
        gop.decode_idx_of_poc[(size_t)pl.poc] = k;
        pic.wctb = wctb;
        pic.hctb = hctb;
        pic.ts_to_rs = ts_to_rs;
        pic.ctb_tile = ctb_tile;
        pic.ctb_slice.assign((size_t)wctb * hctb, 0);
        pic.depth8.assign((size_t)(p.W / 8) * (p.H / 8), 0);
        pic.skip8.assign((size_t)(p.W / 8) * (p.H / 8), 0);
        pic.qp8.assign((size_t)(p.W / 8) * (p.H / 8), 0);
        pic.mode4.assign((size_t)(p.W / 4) * (p.H / 4), 1);
        pic.coeffs.reserve((size_t)p.W * p.H * 3 / 2);
        if (p.extra && k > 0 && (pl.nal_type == 19 || pl.nal_type == 20) && uni(0, 1))
            nal(out, 36, {});   // EOS_NUT before an IDR picture
        pic.code_picture(pl, gop, out, k > 0, param_sets);
        s->slice_type[k] = pic.slice_type;
        s->poc[k] = pl.poc;
        s->output[k] = pl.output ? 1 : 0;
        s->tid[k] = pl.tid;
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
    if (p.extra && uni(0, 1)) nal(out, 37, {});   // EOB_NUT
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
    std::free(s->poc);
    std::free(s->output);
    std::free(s->tid);
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
