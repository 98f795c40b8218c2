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

// Intra schedule entries.  Each intra TU in task order has a dependency list: entries
// without INTRA_DEP_EXTERNAL name a TU of the same CTU by its task index counted from the
// CTU's first; entries with it name a TU of an earlier CTU of the picture by its task
// index in the picture (only a planted test wait is left in that form: the host turns
// each into INTRA_DEP_WATCH | the slot of the CTU's watch list that holds that TU).  A TU
// that some other CTU depends on carries ITU_PUBLISH in reserved[0] of its task-order
// record and publishes its completion in itu_done.
constexpr uint32_t INTRA_DEP_EXTERNAL = 0x80000000u;
constexpr uint32_t INTRA_DEP_WATCH = 0x40000000u;   // | watch slot of the CTU (see ictu_watch)
constexpr uint8_t ITU_PUBLISH = 1u;

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
    // intra CTU tasks (intra.cuh): the CTUs that hold intra TUs in wavefront order (key
    // 2 * row + column), and their TUs ordered by depth in the picture's dependency DAG
    // (task order)
    const int32_t* ictu_addr;            // raster address of intra CTU k
    const int32_t* ictu_tu_off;          // TUs of intra CTU k: task entries [ictu_tu_off[k], [k+1])
    const hevc_tu_t* itu_rec;            // TU records in task order; coeff_offset holds the
                                         // offset of the TU's residual in the CTU's staged ones,
                                         // reserved[0] ITU_PUBLISH
    const int4* itu_res;                 // per task entry: residual source offset (-1: none),
                                         // offset in the CTU's staged residuals, 16-byte chunks
    const uint32_t* itu_dep;             // per task entry: (offset in dep_list << 6) | count
    const uint32_t* dep_list;            // dependency entries (INTRA_DEP_EXTERNAL | index)
    int32_t* itu_done;                   // per task entry: epoch of the launch that completed it
    const uint32_t* ictu_watch;          // per intra CTU: (offset in watch << 8) | count
    const uint32_t* watch;               // TUs of other CTUs each CTU waits for (task indices)
    int32_t n_ictu, n_itu;
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

// Header of a flow area (the intra launches' state of a context or lane): 16 bytes kept
// free; the sticky status word (ST_* bits) follows it, then one CTU ticket counter per
// picture of a launch.
struct FlowState {
    int32_t reserved[4];
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
