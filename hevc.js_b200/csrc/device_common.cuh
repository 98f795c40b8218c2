// device_common.cuh — device-side picture descriptors, tables and helpers shared by the
// reconstruction kernels.
#pragma once

#include <cstdint>

#include "hevcgpu.h"

namespace hevcgpu {

// ---------------------------------------------------------------------------------------
// Per-picture descriptor.  Kernels take an array of these and work items that carry the
// index of their picture, so one launch can serve one picture (plain form) or many
// pictures of many streams (batched form).  All three planes of a picture buffer live in
// one allocation: Cb at y + off_cb, Cr at y + off_cr, with row pitches pitch_y / pitch_c.
// ---------------------------------------------------------------------------------------
struct MotionEnt {           // 4x4 motion grid entry (PUMotionInfo, inter_prediction.h:16)
    int16_t mv[2][2];
    int8_t  ref[2];          // refIdxLX, -1 when predFlagLX is 0
    int16_t pad;
};
static_assert(sizeof(MotionEnt) == 12, "MotionEnt is written as three words by the MC kernel");

// One level of an intra CTU task, packed in 8 bytes (staged into shared memory):
// req(d) > 0 means "dependency slot d must have completed req(d) levels before this level
// runs" (only where the requirement rises); publish means other CTUs wait for this level's
// completion; end is the first task entry of the next level, counted from the CTU's first.
// Fields of 10 bits: x = req(0) | req(1) << 10 | req(2) << 20 | publish << 31,
// y = req(3) | end << 10.
struct IntraLevel {
    uint32_t x, y;
};
constexpr uint32_t INTRA_LEVEL_PUBLISH = 0x80000000u;
constexpr int INTRA_FIELD_MAX = 1023;
__host__ __device__ __forceinline__ int intra_req(const IntraLevel& e, int d) {
    return (int)((d < 3 ? e.x >> (10 * d) : e.y) & 0x3FFu);
}
__host__ __device__ __forceinline__ int intra_end(const IntraLevel& e) { return (int)((e.y >> 10) & 0x3FFu); }

struct PicDesc {
    int32_t width, height;               // luma
    int32_t pitch_y, pitch_c;
    int64_t off_cb, off_cr;
    uint8_t* rec;                        // reconstruction / deblocking buffer
    uint8_t* dst;                        // DPB slot written by SAO
    const uint8_t* ref[2][16];           // reference pictures by list entry (Y base)
    int32_t num_ref[2];
    int32_t ref_poc[2][16];
    const hevc_tu_t* tus;
    const int16_t* coeffs;
    int16_t* resid;                      // residuals of coded intra TUs (at coeff_offset)
    const hevc_pu_t* pus;
    const hevc_wp_t* wp;
    const uint32_t* blk;                 // (W/4)*(H/4)
    MotionEnt* mot;                      // (W/4)*(H/4), built on the device from pus
    const hevc_sao_t* sao;
    const uint8_t* ctb_slice;            // may be null
    const uint16_t* ctb_tile;            // may be null
    const hevc_slice_t* slices;
    const hevc_scaling_t* scaling;       // scaling lists, or null for flat scaling
    // intra CTU tasks (intra.cuh): the CTUs that hold intra TUs, raster order, and their
    // TUs ordered by level of the CTU-local dependency DAG
    const int32_t* ictu_addr;            // raster address of intra CTU k
    const int32_t* ictu_deps;            // 4 per intra CTU: intra CTUs it reads from, or -1
    const int32_t* ictu_tu_off;          // TUs of intra CTU k: itu[ictu_tu_off[k] .. [k+1])
    const hevc_tu_t* itu_rec;            // TU records in task order; coeff_offset holds the
                                         // offset of the TU's residual in the CTU's staged ones
    const int4* itu_res;                 // per task entry: residual source offset (-1: none),
                                         // offset in the CTU's staged residuals, 16-byte chunks
    const int32_t* ictu_lvl_off;         // levels of intra CTU k: ictu_lvl[ictu_lvl_off[k] ..]
    const IntraLevel* ictu_lvl;
    int32_t* ictu_done;                  // per intra CTU: (epoch << 16) | levels completed
    int32_t n_ictu;
    int32_t num_pus;
    int32_t num_slices;
    int32_t log2_ctb, wctb, hctb;
    int32_t sao_enabled;
    int32_t pcm_lf_disabled;
    int32_t strong_intra;
    int32_t intra_smoothing_disabled;
    int32_t cb_qp_offset, cr_qp_offset;
    int32_t tiles_check;                 // tiles enabled and no filtering across tiles
    int32_t slice_check;                 // more than one slice in the picture
    int32_t pcm_bypass_any;              // some CU is PCM or transquant-bypass
};

// Work items ----------------------------------------------------------------------------
// Residual items are TU indices (int32); motion-compensation items are packed strips (mc_item, mc.cuh).

// A launch covers up to MAX_SEGS pictures.  Segment k owns the blocks
// [block0, next block0) of an item-list launch, or blockIdx.y == k of a per-picture
// launch.  The table is a kernel parameter, so a batched launch needs no device-side
// bookkeeping and is captured by value in a CUDA graph.
constexpr int MAX_SEGS = 64;
struct Seg {
    const void* items;
    const PicDesc* pic;
    int32_t n_items;
    int32_t block0;
    int32_t aux0, aux1;   // per-launch extras (intra arming: queue offsets)
};
struct SegTable {
    int32_t n;
    int32_t pad;
    Seg s[MAX_SEGS];
};

__device__ __forceinline__ int find_seg(const SegTable& st, int b) {
    int k = 0;
    while (k + 1 < st.n && st.s[k + 1].block0 <= b) k++;
    return k;
}

// Residual destinations.
enum ResMode : int32_t {
    RES_PACKED = 0,   // pred/out packed per TU at coeff_offset (config-1 form)
    RES_PICTURE = 1,  // inter TUs: add to rec; intra TUs: int16 residual into resid
};

// Device status word bits (written with atomicOr; read by the host after a sync).
enum : uint32_t {
    ST_BAD_RECORD = 1u,   // a record pointed outside its picture; the item was skipped
    ST_TIMEOUT = 2u,      // a bounded wait gave up; the kernel returned early
};

// Shared state of one intra dataflow launch (see intra.cuh).
struct FlowState {
    int32_t head;         // next queue slot to claim
    int32_t tail;         // next queue slot to publish
    uint32_t status;      // ST_* bits
    int32_t pad;
};

__device__ __forceinline__ int clip3(int lo, int hi, int v) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ int clip_u8(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }

// 8-bit z-order address of a 4x4 unit inside a CTU (bit-interleave of 4-bit x, y).
__device__ __forceinline__ uint32_t zorder16(uint32_t bx, uint32_t by) {
    bx = (bx | (bx << 2)) & 0x33u;
    bx = (bx | (bx << 1)) & 0x55u;
    by = (by | (by << 2)) & 0x33u;
    by = (by | (by << 1)) & 0x55u;
    return bx | (by << 1);
}

}  // namespace hevcgpu
