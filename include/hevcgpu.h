/*
 * hevcgpu.h — C ABI of the B200 reconstruction back end for the hevc.js decoder.
 *
 * The host decoder (hevc.js src/bitstream, src/syntax, CABAC in src/decoding) keeps
 * parsing.  Everything it used to do with samples crosses this boundary as plain
 * records: transform blocks with their coefficient levels, prediction units with
 * motion vectors, a 4x4 grid of deblocking side information, SAO parameters per CTU.
 * The GPU side runs dequantisation + inverse transform, intra prediction, motion
 * compensation with weighted prediction, deblocking and SAO, and keeps the decoded
 * picture buffer (DPB) in HBM.
 *
 * Reference interfaces replaced (paths inside privaloops/hevc.js):
 *   perform_dequant            src/decoding/transform.cpp:293
 *   perform_transform_inverse  src/decoding/transform.cpp:374
 *   reconstruct_block          src/decoding/coding_tree.cpp:371
 *   perform_intra_prediction   src/decoding/intra_prediction.cpp:428
 *   perform_inter_prediction   src/decoding/interpolation.cpp:306
 *   apply_deblocking           src/filters/deblocking.cpp:357
 *   apply_sao                  src/filters/sao.cpp:20
 *   Picture / DPB sample store src/common/picture.h:12, src/decoding/dpb.cpp:367
 *
 * Conventions.
 *   - Every function returns HEVCGPU_OK (0) or a negative HEVCGPU_E* code; the text of
 *     the last error of the calling thread is returned by hevcgpu_last_error().
 *   - Host sample planes are 8-bit and tightly packed I420: Y (W*H), Cb, Cr ((W/2)*(H/2)
 *     each), the layout of Picture::write_yuv (src/common/picture.cpp:42) for 8-bit.
 *   - Only 8-bit 4:2:0 is accepted (HEVCGPU_EUNSUPPORTED otherwise).
 *   - No function falls back to a CPU implementation: without a usable CUDA device the
 *     create call fails with HEVCGPU_ECUDA.
 */
#ifndef HEVCGPU_H
#define HEVCGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HEVCGPU_ABI_VERSION 2

/* ---- status codes (negative values map to HEVC_ERROR of src/wasm/hevc_api.h:43) ---- */
#define HEVCGPU_OK            0
#define HEVCGPU_EINVAL       -1   /* bad argument or record outside the picture        */
#define HEVCGPU_ECUDA        -2   /* CUDA runtime error (message has the CUDA string)  */
#define HEVCGPU_ENOMEM       -3   /* device or pinned host allocation failed / budget */
#define HEVCGPU_EUNSUPPORTED -4   /* bit depth, chroma format or tool not supported    */
#define HEVCGPU_ETIMEOUT     -5   /* a bounded device wait gave up (status word set)   */
#define HEVCGPU_EDEVICE      -6   /* a kernel reported a record it refused (bounds)    */

/* ---- record layouts (all little-endian, naturally aligned, no padding surprises) ---- */

/* Transform block flags. */
#define HEVC_TU_INTRA   0x01  /* CuPredMode == MODE_INTRA: predicted by intra_mode       */
#define HEVC_TU_CODED   0x02  /* has coefficient levels at coeff_offset (cbf set)        */
#define HEVC_TU_TSKIP   0x04  /* transform_skip_flag                                    */
#define HEVC_TU_BYPASS  0x08  /* cu_transquant_bypass: levels are the residual          */
#define HEVC_TU_PCM     0x10  /* pcm_flag: the levels are the samples, no prediction     */
                              /* (coding_tree.cpp:1425-1469; with INTRA and CODED)      */

/* One transform block of one colour component (decode order = z-scan, luma before
 * chroma, 4x4-luma chroma deferred to blkIdx 3; src/decoding/coding_tree.cpp:1256). */
typedef struct hevc_tu {
    uint16_t x, y;          /* top-left in samples of component c_idx                  */
    uint8_t  log2_size;     /* 2..5                                                    */
    uint8_t  c_idx;         /* 0 = Y, 1 = Cb, 2 = Cr                                   */
    uint8_t  qp;            /* qP' = QpY + QpBdOffsetY, or the mapped chroma qP'       */
    uint8_t  flags;         /* HEVC_TU_*                                               */
    uint8_t  intra_mode;    /* 0..34, for HEVC_TU_INTRA                                */
    uint8_t  reserved[3];
    uint32_t coeff_offset;  /* first int16 of this block's N*N row-major levels       */
} hevc_tu_t;                /* 16 bytes */

/* One prediction unit (src/decoding/coding_tree.cpp:882-953).  List l is used when
 * ref_idx[l] >= 0 (predFlagLX); ref_idx indexes the picture's reference list. */
typedef struct hevc_pu {
    uint16_t x, y;          /* luma top-left                                           */
    uint8_t  w, h;          /* luma size, 4..64                                        */
    int8_t   ref_idx[2];    /* refIdxL0, refIdxL1 (-1: list unused)                    */
    int16_t  mv[2][2];      /* quarter-pel luma MV: mv[list][0] = x, mv[list][1] = y   */
    int16_t  wp;            /* -1: default weighted prediction; else row of the WP table */
    uint16_t reserved;
} hevc_pu_t;                /* 20 bytes */

/* Explicit weighted prediction parameters of one PU class, already resolved from the
 * slice's pred_weight_table for its (refIdxL0, refIdxL1): weighted_pred_explicit,
 * src/decoding/interpolation.cpp:246. */
typedef struct hevc_wp {
    int16_t log2wd[2];      /* log2Wd for luma [0] and chroma [1] (denominator + shift1) */
    int16_t w[2][3];        /* weight [list][component]                                 */
    int16_t o[2][3];        /* offset [list][component], already << (BitDepth - 8)      */
} hevc_wp_t;                /* 28 bytes */

/* 4x4-luma-block side information word (deblocking grids of DecodingContext,
 * src/decoding/coding_tree.h:65-70 and CUInfo :21-30). */
#define HEVC_BLK_EDGE_V   0x01u   /* edge_flags_v: vertical TU/PU/CU edge at left side  */
#define HEVC_BLK_EDGE_H   0x02u   /* edge_flags_h: horizontal edge at top side          */
#define HEVC_BLK_CBF      0x04u   /* cbf_luma of the covering luma TU                   */
#define HEVC_BLK_INTRA    0x08u   /* CU is intra                                        */
#define HEVC_BLK_PCM      0x10u   /* CU is PCM                                          */
#define HEVC_BLK_BYPASS   0x20u   /* cu_transquant_bypass                               */
#define HEVC_BLK_TU_SHIFT 8       /* bits 8..15: log2 of the covering TU size           */
#define HEVC_BLK_QP_SHIFT 16      /* bits 16..23: QpY of the CU, two's complement int8  */

/* SAO parameters of one CTU (DecodingContext::SaoParams, coding_tree.h:73-78). */
typedef struct hevc_sao {
    uint8_t type[3];        /* 0 off, 1 band offset, 2 edge offset                     */
    uint8_t band_pos[3];    /* sao_band_position                                       */
    uint8_t eo_class[3];    /* sao_eo_class                                            */
    int8_t  offset[3][5];   /* SaoOffsetVal in the reference layout: EO [+,+,0,-,-],   */
                            /* BO [o0,o1,o2,o3,0] (coding_tree.cpp:146-164)            */
} hevc_sao_t;               /* 24 bytes */

/* Per-slice filter parameters (SliceHeader fields read by apply_deblocking/apply_sao). */
typedef struct hevc_slice {
    int8_t  beta_offset_div2;
    int8_t  tc_offset_div2;
    uint8_t deblocking_disabled;      /* slice_deblocking_filter_disabled_flag          */
    uint8_t lf_across_slices;         /* slice_loop_filter_across_slices_enabled_flag   */
} hevc_slice_t;

/* Scaling lists of the active parameter set: ScalingListData (src/syntax/sps.h:15-31),
 * i.e. pps.scaling_list_data when pps_scaling_list_data_present_flag, else
 * sps.scaling_list_data, exactly as the parser stores them (set_defaults and parse,
 * src/syntax/sps.cpp:41-113).  perform_dequant (src/decoding/transform.cpp:320-358) reads
 * list[sizeId][matrixId] at y*4+x for 4x4 blocks and at (y/r)*8 + x/r (r = N/8) above,
 * with dc[sizeId-2][matrixId] (0 read as 16) at (0,0) of 16x16 and 32x32 blocks;
 * matrixId = c_idx + 3 * !intra below 32x32 and 3 * !intra at 32x32. */
typedef struct hevc_scaling {
    uint8_t list[4][6][64];   /* ScalingListData::scaling_list                        */
    uint8_t dc[2][6];         /* ScalingListData::scaling_list_dc                     */
    uint8_t reserved[4];
} hevc_scaling_t;             /* 1552 bytes */

/* Picture-level parameters (SPS/PPS/slice fields the reconstruction reads). */
typedef struct hevc_pic_params {
    int32_t width, height;            /* luma samples, multiples of 8                   */
    int32_t bit_depth;                /* 8                                              */
    int32_t log2_ctb;                 /* CtbLog2SizeY, 4..6                             */
    int32_t log2_min_cb;              /* MinCbLog2SizeY                                 */
    int32_t log2_min_tb;              /* MinTbLog2SizeY (2)                             */
    int32_t strong_intra_smoothing;   /* strong_intra_smoothing_enabled_flag            */
    int32_t intra_smoothing_disabled; /* intra_smoothing_disabled_flag                  */
    int32_t pcm_loop_filter_disabled; /* pcm_loop_filter_disabled_flag                  */
    int32_t sao_enabled;              /* sample_adaptive_offset_enabled_flag            */
    int32_t cb_qp_offset, cr_qp_offset;   /* pps_cb_qp_offset, pps_cr_qp_offset         */
    int32_t tiles_enabled;            /* ctb_tile is meaningful                         */
    int32_t loop_filter_across_tiles; /* loop_filter_across_tiles_enabled_flag          */
    int32_t num_ref[2];               /* entries in RefPicList0/1                       */
    int32_t ref_poc[2][16];           /* POC of each entry (deblocking Bs compares POCs) */
    int32_t ref_slot[2][16];          /* DPB slot of each entry (picture API)           */
} hevc_pic_params_t;

/* Everything one picture hands to the GPU at its end (the point where
 * src/decoding/decoder.cpp:270 calls apply_deblocking today). */
typedef struct hevc_picture_syntax {
    hevc_pic_params_t   params;
    int32_t             num_tus;      /* intra TUs (coded or not) + coded inter TUs     */
    const hevc_tu_t*    tus;          /* in decode order                                */
    uint64_t            num_coeffs;
    const int16_t*      coeffs;
    int32_t             num_pus;
    const hevc_pu_t*    pus;
    int32_t             num_wp;
    const hevc_wp_t*    wp;
    const uint32_t*     blk;          /* (width/4)*(height/4) HEVC_BLK_* words          */
    const hevc_sao_t*   sao;          /* PicSizeInCtbsY entries, raster order           */
    const uint8_t*      ctb_slice;    /* slice index per CTB (raster), or NULL = all 0  */
    const uint16_t*     ctb_tile;     /* TileId per CTB (raster), or NULL               */
    int32_t             num_slices;
    const hevc_slice_t* slices;
    const hevc_scaling_t* scaling;    /* NULL: flat scaling (scaling_list_enabled_flag = 0) */
} hevc_picture_syntax_t;

/* ---- context ---- */
typedef struct hevcgpu_ctx hevcgpu_ctx_t;
typedef struct hevcgpu_stream hevcgpu_stream_t;
typedef struct hevcgpu_job hevcgpu_job_t;

int         hevcgpu_abi_version(void);
const char* hevcgpu_last_error(void);
int         hevcgpu_create(int device, hevcgpu_ctx_t** out);
void        hevcgpu_destroy(hevcgpu_ctx_t* ctx);
int         hevcgpu_sync(hevcgpu_ctx_t* ctx);

/* ---- stage entry points on host memory (synchronous; copies inside) ---- */

/* Dequant + inverse DST/DCT + add prediction + clip for independent blocks.
 * Replaces perform_dequant (transform.cpp:293), perform_transform_inverse
 * (transform.cpp:374) and reconstruct_block (coding_tree.cpp:371).  Block t reads its
 * N*N levels at coeffs + tus[t].coeff_offset, its N*N prediction samples at
 * pred + tus[t].coeff_offset and writes N*N samples at out + tus[t].coeff_offset. */
int hevcgpu_residual_blocks(hevcgpu_ctx_t* ctx, const hevc_tu_t* tus, int32_t num_tus,
                            const int16_t* coeffs, uint64_t num_coeffs,
                            const uint8_t* pred, uint8_t* out);

/* The same with scaling lists (sps.scaling_list_enabled_flag = 1): each block dequantises
 * with the matrix of its size, plane and HEVC_TU_INTRA flag (CuPredMode of the CU at the
 * block, transform.cpp:330-336).  scaling NULL is flat, as hevcgpu_residual_blocks. */
int hevcgpu_residual_blocks_scaled(hevcgpu_ctx_t* ctx, const hevc_scaling_t* scaling,
                                   const hevc_tu_t* tus, int32_t num_tus,
                                   const int16_t* coeffs, uint64_t num_coeffs,
                                   const uint8_t* pred, uint8_t* out);

/* Motion-compensated prediction of every PU into out (I420, params->width x height).
 * refs[i] is the I420 picture for reference-list slot i (params->ref_slot values
 * index this array).  Replaces perform_inter_prediction (interpolation.cpp:306) and
 * the sample store of coding_tree.cpp:892-922. */
int hevcgpu_inter_pred(hevcgpu_ctx_t* ctx, const hevc_pic_params_t* params,
                       const hevc_pu_t* pus, int32_t num_pus,
                       const hevc_wp_t* wp, int32_t num_wp,
                       const uint8_t* const* refs, int32_t num_refs, uint8_t* out);

/* In-loop filters of one reconstructed picture: deblocking (apply_deblocking,
 * deblocking.cpp:357) when do_deblock, then SAO (apply_sao, sao.cpp:20) when do_sao.
 * syn->tus/coeffs are not used; syn->pus provide motion for the Bs derivation. */
int hevcgpu_loop_filter(hevcgpu_ctx_t* ctx, const hevc_picture_syntax_t* syn,
                        const uint8_t* in, uint8_t* out, int do_deblock, int do_sao);

/* Intra prediction + residual for the intra TUs of syn over an I420 picture that
 * already holds every inter sample (in/out may alias).  Replaces
 * perform_intra_prediction (intra_prediction.cpp:428) in its TU loop. */
int hevcgpu_intra_recon(hevcgpu_ctx_t* ctx, const hevc_picture_syntax_t* syn,
                        const uint8_t* in, uint8_t* out);

/* Whole-picture reconstruction (MC, residual, intra wavefront, deblocking, SAO) of one
 * picture; refs as in hevcgpu_inter_pred. */
int hevcgpu_reconstruct_picture(hevcgpu_ctx_t* ctx, const hevc_picture_syntax_t* syn,
                                const uint8_t* const* refs, int32_t num_refs,
                                uint8_t* out);

/* ---- decoded picture buffer in HBM + picture pipeline ---- */

/* A stream owns num_slots DPB slots of width x height 8-bit 4:2:0 in HBM plus the work
 * buffers of one picture in flight.  Admission: fails with HEVCGPU_ENOMEM when the
 * context's HBM budget (hevcgpu_set_budget) would be exceeded. */
int  hevcgpu_set_budget(hevcgpu_ctx_t* ctx, uint64_t bytes);
uint64_t hevcgpu_bytes_in_use(hevcgpu_ctx_t* ctx);
int  hevcgpu_stream_open(hevcgpu_ctx_t* ctx, int32_t width, int32_t height,
                         int32_t bit_depth, int32_t num_slots, hevcgpu_stream_t** out);
void hevcgpu_stream_close(hevcgpu_stream_t* st);
int  hevcgpu_slot_upload(hevcgpu_stream_t* st, int32_t slot, const uint8_t* i420);
int  hevcgpu_slot_download(hevcgpu_stream_t* st, int32_t slot, uint8_t* i420);

/* Conformance window in luma samples: conf_win_*_offset times SubWidthC / SubHeightC, as
 * the reference's Picture keeps it (src/wasm/hevc_api.cpp:58-65); even values for 4:2:0. */
typedef struct hevc_crop {
    int32_t left, right, top, bottom;
} hevc_crop_t;

/* A slot as hevc_decoder_get_frame hands a picture out (src/wasm/hevc_api.cpp:49-77,
 * HEVCFrame of src/wasm/hevc_api.h:21-33): the samples inside the conformance window as
 * 16-bit planes.  Writes (W - left - right) x (H - top - bottom) samples to y (row
 * stride stride_y samples) and half of each to cb and cr (stride_c).  crop NULL is the
 * whole picture.  The widening runs on the device; the call returns when the planes have
 * landed.  Replaces the frame copy a caller of hevc_decoder_get_frame makes. */
int  hevcgpu_slot_download_frame(hevcgpu_stream_t* st, int32_t slot, const hevc_crop_t* crop,
                                 uint16_t* y, int32_t stride_y, uint16_t* cb, uint16_t* cr,
                                 int32_t stride_c);
/* The checksum of the H.265 decoded picture hash SEI (Rec. ITU-T H.265 D.3.19) of each plane
 * of the frame hevcgpu_slot_download_frame would hand out (the same conformance window,
 * with x and y counted from its top-left corner): out[0..2] = Y, Cb, Cr, each the sum
 * modulo 2^32 of sample ^ ((x & 0xFF) ^ (y & 0xFF) ^ (x >> 8) ^ (y >> 8)).  Computed on the
 * device; only the three words come back, so a decoder checks a frame against a picture
 * hash (or a test against its oracle) without copying the frame.  The reference carries
 * no such call: it checks frames by MD5 of the whole output on the host
 * (tools/oracle_test.sh). */
int  hevcgpu_slot_checksum(hevcgpu_stream_t* st, int32_t slot, const hevc_crop_t* crop,
                           uint32_t* out);
/* Device address of a slot's Y plane and the row pitches (for zero-copy consumers). */
int  hevcgpu_slot_device_ptr(hevcgpu_stream_t* st, int32_t slot, void** y, void** cb,
                             void** cr, int32_t* pitch_y, int32_t* pitch_c);

/* Prepare a picture: host-side packing (bins, per-CTU intra lists) and one upload of
 * the records into device memory owned by the job.  The job can be launched many
 * times (benchmarks) and is freed with hevcgpu_job_free.  The large record arrays (TUs,
 * coefficient levels, PUs, 4x4 grid) are packed into pinned staging and uploaded from
 * there; an array that already lies in page-locked memory is uploaded from where it
 * lies, with no staging copy. */
int  hevcgpu_job_prepare(hevcgpu_stream_t* st, const hevc_picture_syntax_t* syn,
                         hevcgpu_job_t** out);
void hevcgpu_job_free(hevcgpu_job_t* job);
/* Bytes the prepare call copied host -> device for this job (records + work lists). */
uint64_t hevcgpu_job_upload_bytes(hevcgpu_job_t* job);
/* Page-locked host memory for a recorder's record arrays (the per-picture data the
 * reference keeps in DecodingContext, decoding/coding_tree.h:60-78, recorded as TU, PU and
 * grid arrays): arrays in it are uploaded without a staging copy.  Any CUDA device of the
 * process may be current. */
int  hevcgpu_host_alloc(size_t bytes, void** out);
int  hevcgpu_host_free(void* p);
/* Plain form: one launch per stage for this picture, into DPB slot dst_slot, reading
 * reference slots from params.ref_slot.  Asynchronous on the stream's CUDA stream. */
int  hevcgpu_job_launch(hevcgpu_job_t* job, int32_t dst_slot);
/* Batched form: the stages of n pictures (any streams of one context, no picture may
 * reference another picture of the same batch) run as merged launches. */
int  hevcgpu_batch_launch(hevcgpu_job_t* const* jobs, const int32_t* dst_slots, int32_t n);
int  hevcgpu_stream_sync(hevcgpu_stream_t* st);

/* Lanes: launch queues of one context that run side by side on the device.  A lane has
 * its own CUDA stream and its own intra-task state, so batches launched on different
 * lanes overlap (one batch's latency-bound intra waves share the SMs with another's MC
 * and filters) - the device side of continuous batching.  No counterpart in the
 * reference, whose decoder reconstructs one picture at a time (decoder.cpp:52-304).
 * Ordering: a lane batch starts after everything queued so far on the context's stream
 * (record uploads, slot uploads), and a job launched on a lane other than its last one
 * waits for that launch.  A picture that references a slot written by a batch of another
 * lane must be launched after hevcgpu_lane_sync of that lane (or on the same lane); the
 * context's own slot downloads likewise follow hevcgpu_lane_sync.  A lane is used from
 * one host thread at a time. */
typedef struct hevcgpu_lane hevcgpu_lane_t;
int   hevcgpu_lane_open(hevcgpu_ctx_t* ctx, hevcgpu_lane_t** out);
void  hevcgpu_lane_close(hevcgpu_lane_t* lane);
int   hevcgpu_lane_batch_launch(hevcgpu_lane_t* lane, hevcgpu_job_t* const* jobs,
                                const int32_t* dst_slots, int32_t n);
/* Waits for the lane and returns its device status (HEVCGPU_ETIMEOUT / EDEVICE). */
int   hevcgpu_lane_sync(hevcgpu_lane_t* lane);
/* CUDA stream (cudaStream_t) of the lane. */
void* hevcgpu_lane_cuda_stream(hevcgpu_lane_t* lane);
/* CUDA stream (cudaStream_t) the lane's asynchronous downloads run on: a caller records an
 * event there after hevcgpu_lane_slots_download_async to learn on the device when the
 * frames landed (the serving loop's latency ends there). */
void* hevcgpu_lane_copy_stream(hevcgpu_lane_t* lane);
/* hevcgpu_slots_download with the copies queued on the lane, after its batches: the
 * pictures of a lane batch can be read back without waiting for the other lanes.
 * Returns the lane's device status, like hevcgpu_lane_sync. */
int   hevcgpu_lane_slots_download(hevcgpu_lane_t* lane, hevcgpu_stream_t* const* sts,
                                  const int32_t* slots, int32_t n, uint8_t* const* outs);
/* The same copies without waiting: they run on the lane's own copy stream after the work
 * queued on the lane so far, so the lane's next batches do not wait for them; a later
 * launch or upload that writes one of these slots waits for their copies on the device.
 * Every destination must be page-locked host memory (cudaHostAlloc / cudaHostRegister),
 * which the copies write directly.  *ticket identifies the download; the frames are
 * complete once hevcgpu_lane_wait(lane, ticket) has returned (or after hevcgpu_lane_sync).  A
 * decoder pipeline overlaps the copies of one batch with the preparation of the next
 * (the reference hands each frame out synchronously: hevc_decoder_get_frame,
 * wasm/hevc_api.h:63). */
int   hevcgpu_lane_slots_download_async(hevcgpu_lane_t* lane, hevcgpu_stream_t* const* sts,
                                        const int32_t* slots, int32_t n, uint8_t* const* outs,
                                        uint64_t* ticket);
/* Waits until the download with this ticket has landed; returns the lane's device status,
 * like hevcgpu_lane_sync. */
int   hevcgpu_lane_wait(hevcgpu_lane_t* lane, uint64_t ticket);

/* Batched host-side calls for a decoder that finishes several pictures at once (one per
 * stream).  The work is spread over the context's host worker threads (one per
 * hardware thread, started on first use).
 *
 * hevcgpu_jobs_prepare: hevcgpu_job_prepare of syns[i] on sts[i] for i < n (streams of
 * one context).  On failure no job is returned (every out[i] is null) and the message
 * names the first failing picture.
 * hevcgpu_slots_download: slot slots[i] of sts[i] into the I420 host buffer outs[i].
 * Pageable buffers are filled from pinned staging as each picture's copy lands; pinned
 * buffers (cudaHostAlloc / cudaHostRegister) receive the copy directly.  Returns when
 * every buffer is written.  Together with hevcgpu_batch_launch these serve, for a batch,
 * what the reference's frame output hands to its caller per picture
 * (Decoder::output_pictures, decoding/decoder.cpp:320; hevc_decoder_get_frame,
 * wasm/hevc_api.cpp:49), as packed I420 host frames. */
int  hevcgpu_jobs_prepare(hevcgpu_stream_t* const* sts, const hevc_picture_syntax_t* const* syns,
                          int32_t n, hevcgpu_job_t** out);

/* hevcgpu_jobs_prepare without waiting for the copies of the caller's page-locked arrays:
 * it returns once the jobs are built, with those copies still in flight (arrays in
 * pageable memory were copied to staging, so they may change at once).  Before it writes
 * into a page-locked array of a picture again, the caller waits for that picture's job
 * with hevcgpu_job_wait_uploaded; launching, downloading and freeing the jobs need no
 * wait.  A recorder that fills several page-locked record buffers in turn uses this to
 * overlap a batch's transfer with the building of the next. */
int  hevcgpu_jobs_prepare_async(hevcgpu_stream_t* const* sts, const hevc_picture_syntax_t* const* syns,
                                int32_t n, hevcgpu_job_t** out);
/* Returns once the copies of a job's page-locked record arrays have read them. */
int  hevcgpu_job_wait_uploaded(hevcgpu_job_t* job);

/* Test hook for the device timeout path (no counterpart in the reference): the first task
 * of the job's intra schedule is made to wait for its own completion, which it can never
 * publish.  Its bounded wait gives up after about a second, the kernel returns, and the
 * next sync reports HEVCGPU_ETIMEOUT; the context stays usable.  The injection is a change
 * of the job's uploaded schedule on the host side: nothing faults or traps.
 * HEVCGPU_EINVAL for a job without intra TUs. */
int  hevcgpu_job_plant_unmet_wait(hevcgpu_job_t* job);

/* The intra schedule the back end builds for a picture (no counterpart in the reference;
 * host work only, no device is needed), for tools and tests: the CTUs that hold intra TUs
 * in the order CTAs take them (wavefront order, key 2 * row + column), each CTU's tasks
 * (its intra TUs, every one after the TUs it depends on), each task's dependency list and
 * each CTU's watch list (the TUs of earlier CTUs it waits for).  A dependency entry is the
 * index of a task of the same CTU counted from the CTU's first, or
 * HEVC_INTRA_DEP_WATCH | the slot of the CTU's watch list.  The arrays belong to the
 * calling thread and stay valid until its next call. */
#define HEVC_INTRA_DEP_WATCH 0x40000000u
#define HEVC_INTRA_PUBLISH 1u          /* task_flags: a TU of another CTU depends on it */
typedef struct hevc_intra_schedule {
    int32_t n_ctu, n_task, n_dep, n_watch;
    const int32_t*  ctu_addr;      /* n_ctu: raster address of each CTU, in task order     */
    const int32_t*  ctu_first;     /* n_ctu + 1: first task of each CTU                    */
    const int32_t*  task_tu;       /* n_task: the task's TU (index into syn->tus)          */
    const uint32_t* task_deps;     /* n_task: (offset into deps << 6) | number of entries  */
    const uint32_t* deps;          /* n_dep dependency entries                             */
    const uint8_t*  task_flags;    /* n_task: HEVC_INTRA_PUBLISH                           */
    const uint32_t* ctu_watch;     /* n_ctu: (offset into watch << 8) | number of slots    */
    const uint32_t* watch;         /* n_watch: the watched TUs, as task indices            */
} hevc_intra_schedule_t;
int  hevcgpu_intra_schedule(const hevc_picture_syntax_t* syn, hevc_intra_schedule_t* out);

/* The motion-compensation work lists the back end builds for a picture (no counterpart in
 * the reference; host work only), for tools and tests: one item per strip of 4 columns and
 * up to 16 rows of one PU in one plane, luma and chroma lists.  Item bits: 0-19 the PU,
 * 20-23 the strip's column / 4, 24-25 its first row / 16, 26-28 its rows / 4 - 1 (luma) or
 * rows / 2 - 1 (chroma), 29 the chroma plane (0 Cb, 1 Cr).  Each list is ordered by class:
 * bi-predicted strips first, then strips whose reference windows lie inside the picture,
 * then taller strips first.  The arrays belong to the calling thread and stay valid until
 * its next call. */
int  hevcgpu_mc_strips(const hevc_picture_syntax_t* syn, const uint32_t** luma, int32_t* n_luma,
                       const uint32_t** chroma, int32_t* n_chroma);
int  hevcgpu_slots_download(hevcgpu_stream_t* const* sts, const int32_t* slots, int32_t n,
                            uint8_t* const* outs);
/* CUDA stream (cudaStream_t) the context launches on. */
void* hevcgpu_cuda_stream(hevcgpu_ctx_t* ctx);
/* Number of kernel launches issued by this context so far. */
uint64_t hevcgpu_launch_count(hevcgpu_ctx_t* ctx);

/* Stage profiling: when enabled, CUDA events are recorded on the context's stream around
 * each reconstruction stage of every later launch.  hevcgpu_profile_read waits for the
 * stream and returns, per stage, the summed device milliseconds and the number of kernel
 * launches since the previous read.  Stages: 0 motion grid, 1 motion compensation,
 * 2 residual, 3 intra wavefront, 4 deblocking (vertical edges), 5 deblocking
 * (horizontal edges), 6 SAO. */
#define HEVCGPU_NUM_STAGES 7
int hevcgpu_profile_enable(hevcgpu_ctx_t* ctx, int enable);
int hevcgpu_profile_read(hevcgpu_ctx_t* ctx, double* ms, uint64_t* launches);

/* End-to-end decode-side call: prepare + upload + launch + wait for one picture. */
int  hevcgpu_picture_decode(hevcgpu_stream_t* st, const hevc_picture_syntax_t* syn,
                            int32_t dst_slot);

/* Residual blocks with no allocation.  No counterpart in the reference: same blocks and
 * results as hevcgpu_residual_blocks (flat dequantisation: scaling lists are not offered
 * here), for callers that must not allocate while decoding (a serving process that sized
 * its device memory once at start-up; decode threads on which cudaMalloc/cudaFree would
 * synchronise the device and stall other streams).  tus is a host array; d_coeffs
 * (num_coeffs int16 levels), d_pred and d_out (num_coeffs bytes each) are caller-owned
 * DEVICE buffers of ctx's device, 16-byte aligned.  The call allocates no memory: its
 * scratch is a fixed static device array sized for HEVCGPU_STATIC_MAX_TUS blocks, and more
 * blocks are rejected with HEVCGPU_EINVAL; so are devices numbered 16 and above.  Runs on
 * ctx's stream and returns once d_out is written.  The first call on each device looks up
 * the scratch address (and may load the module on that device): make it before any stream
 * capture begins.  All calls on one device share that device's scratch, so a lock per
 * device serialises them; calls on different devices do not wait for each other. */
#define HEVCGPU_STATIC_MAX_TUS 65536
int  hevcgpu_residual_blocks_static(hevcgpu_ctx_t* ctx, const hevc_tu_t* tus, int32_t num_tus,
                                    const int16_t* d_coeffs, uint64_t num_coeffs,
                                    const uint8_t* d_pred, uint8_t* d_out);

#ifdef __cplusplus
}
#endif

#endif /* HEVCGPU_H */
