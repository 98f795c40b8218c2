/* bitgen.h — seeded generator of random-syntax HEVC Main-profile bitstreams.
 *
 * It draws a legal coding tree per CTU (CU splits, intra 2Nx2N / NxN partitions, intra
 * prediction modes, skipped and inter CUs with their partitions (AMP included), merge
 * indices, inter prediction directions, reference indices, motion vector differences and
 * predictor flags, transform trees, coded blocks and their levels, SAO parameters, QPs) and
 * CABAC-encodes it (Rec. ITU-T H.265 clause 9.3: binarisations, context selection and
 * initialisation, arithmetic encoding) into an Annex-B byte stream: VPS, SPS, PPS, then the
 * slice segments of each picture.  An IDR picture comes first, then IDR pictures or P and B
 * pictures, low delay or random access (hierarchical mini-GOPs, reordered for output), with
 * short-term reference picture sets in the slice headers, reference list sizes, TMVP and
 * weighted prediction tables.  Coding tools on request: cu_qp_delta, chroma QP offsets,
 * deblocking control, several (and dependent) slice segments, tiles, WPP with entry points,
 * transquant bypass, transform skip, sign data hiding, PCM, scaling lists.  The reference
 * decoder parses these streams (src/decoding/syntax_elements.cpp, residual_coding.cpp:175,
 * cabac.cpp:38); the records it produces are the ones the generator drew, which
 * tests/test_bitgen.py checks.
 *
 * Host code only; no counterpart in the reference (its streams come from x265/ffmpeg). */
#ifndef HEVC_BITGEN_H
#define HEVC_BITGEN_H

#include <stddef.h>
#include <stdint.h>

#include "hevcgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hevcgen_cfg {
    int32_t  width, height;      /* luma samples, multiples of 8                          */
    uint64_t seed;
    int32_t  pictures;           /* IDR pictures in the stream                            */
    int32_t  log2_ctb;           /* 4..6                                                  */
    double   p_split;            /* CU quadtree split probability (down to 8x8)           */
    double   p_nxn;              /* 8x8 CU split into four 4x4 luma prediction blocks     */
    double   p_tu_split;         /* transform tree split probability (where allowed)      */
    double   p_cbf;              /* coded block flag probability per luma / chroma block  */
    double   p_sig;              /* probability of a nonzero level inside the coded area  */
    int32_t  max_level;          /* largest |level| drawn                                 */
    int32_t  qp_min, qp_max;     /* slice QP range                                        */
    int32_t  sao;                /* SAO enabled (parameters drawn per CTB)                */
    /* inter pictures; inter = 0 makes every picture an IDR picture */
    int32_t  inter;              /* 1: picture 0 is IDR, the others P or B (TRAIL_R)      */
    double   p_b;                /* a non-IDR picture is a B picture (low delay: both     */
                                 /* lists hold earlier pictures)                          */
    int32_t  max_refs;           /* 1..4: the reference picture set keeps the last        */
                                 /* max_refs pictures, each used by the current one or not */
    double   p_intra_cu;         /* an intra CU in a P/B slice                            */
    double   p_skip;             /* cu_skip_flag                                          */
    double   p_merge;            /* merge_flag of a PU of a CU not skipped                */
    int32_t  max_mvd;            /* largest |mvd| component drawn, quarter samples        */
    int32_t  amp;                /* amp_enabled_flag (asymmetric partitions)              */
    int32_t  tmvp;               /* sps_temporal_mvp_enabled_flag (slice flag drawn)      */
    int32_t  max_merge;          /* MaxNumMergeCand 1..5; 0: drawn per slice              */
    int32_t  wp;                 /* weighted_pred_flag and weighted_bipred_flag (tables   */
                                 /* drawn per slice)                                      */
    int32_t  depth_inter;        /* max_transform_hierarchy_depth_inter 0..2              */
    /* coding tools; 0 leaves a tool off */
    int32_t  qp_delta_depth;     /* cu_qp_delta_enabled_flag, diff_cu_qp_delta_depth =    */
                                 /* qp_delta_depth - 1 (at most log2_ctb - 3)             */
    int32_t  chroma_qp_offsets;  /* PPS and slice Cb / Cr QP offsets drawn                */
    int32_t  deblock_ctl;        /* PPS deblocking flags and offsets, slice overrides drawn */
    int32_t  slices;             /* about this many slice segments per picture (more where */
                                 /* tiles or WPP force boundaries)                        */
    int32_t  dependent_slices;   /* dependent_slice_segments_enabled_flag; about half the */
                                 /* segments after the first then continue their slice    */
    int32_t  tile_cols, tile_rows;   /* tiles, within Main's 256 x 64 minimum tile size   */
    int32_t  wpp;                /* entropy_coding_sync_enabled_flag (not with tiles)     */
    double   p_bypass;           /* cu_transquant_bypass_flag                             */
    double   p_tskip;            /* transform_skip_flag of a 4x4 block                    */
    int32_t  sdh;                /* sign_data_hiding_enabled_flag                         */
    double   p_pcm;              /* pcm_flag of a CU of a PCM size (bit depths, sizes and */
                                 /* pcm_loop_filter_disabled_flag drawn)                  */
    int32_t  scaling;            /* 1 default scaling lists, 2 lists in the SPS, 3 in the PPS */
    /* HEVCGEN_QUIRK_* bits: write some tools the way the reference's parser reads them
     * (where it departs from H.265) instead of the way the standard defines them */
    int32_t  ref_quirks;
    int32_t  ra_gop;             /* with inter: 0 or 1 low delay; G > 1 random access, mini-GOPs */
                                 /* of G pictures coded last-first then by bisection (pictures */
                                 /* reordered for output)                                 */
    int32_t  idr_period;         /* an IDR picture every idr_period pictures (POCs restart; */
                                 /* no_output_of_prior_pics_flag drawn); 0: only the first */
    int32_t  crop;               /* a conformance cropping window drawn                   */
    double   p_no_output;        /* pic_output_flag = 0 (output_flag_present_flag set)    */
    int32_t  long_term;          /* long_term_ref_pics_present_flag; with low delay, each */
                                 /* period's IDR picture is a long-term reference from its */
                                 /* third picture on                                      */
    int32_t  list_mod;           /* lists_modification_present_flag (list entries drawn)  */
    int32_t  extra_syntax;       /* syntax a decoder reads past: access unit delimiters,  */
                                 /* prefix and suffix SEI (user data), filler data, end of */
                                 /* sequence / bitstream NAL units, VUI, slice_reserved_flag */
                                 /* bits and slice header extensions                      */
    int32_t  sps_rps;            /* short-term RPSs in the SPS (picked by index in the slice */
                                 /* headers), some coded by inter RPS prediction          */
    int32_t  cra;                /* random access: some mini-GOPs end in a CRA picture   */
                                 /* whose inner pictures are its leading pictures (RASL, */
                                 /* and RADL from the middle one on)                      */
    int32_t  poc_lsb_bits;       /* log2_max_pic_order_cnt_lsb (0: 8); raised where the   */
                                 /* GOP needs more; small values make POCs wrap            */
    int32_t  resize;             /* with idr_period: an IDR picture may bring a new SPS   */
                                 /* (a smaller picture size) and PPS                      */
    int32_t  temporal;           /* random access: temporal sub-layers, TemporalId the    */
                                 /* picture's bisection depth (VPS/SPS sub-layer fields); */
                                 /* TSA and STSA pictures where the plan allows them      */
    int32_t  nonref_types;       /* a picture no later one uses gets TRAIL_N, TSA_N,      */
                                 /* STSA_N, RADL_N or RASL_N (sub-layer non-reference)    */
    int32_t  pps_count;          /* PPSs in the stream (ids 0..): the enabled tools switched */
                                 /* on or off and drawn again per PPS; each picture refers */
                                 /* to one of them                                        */
    int32_t  bit_depth;          /* 8 (0 means 8) or 10: BitDepthY = BitDepthC; with 10,  */
                                 /* CuQpDeltaVal keeps QpY in 0..51, the TU records hold */
                                 /* Qp' (QpY + QpBdOffset), SAO offsets reach 31         */
} hevcgen_cfg_t;

/* Tiles and PCM: after end_of_subset_one_bit and after pcm_flag the reference reads an
 * alignment bit equal to one although the arithmetic code's flush already ends in it, so it
 * skips a byte when the flush ends on a byte boundary (coding_tree.cpp:628-632, :1432); it
 * does not initialise the context variables at the first CTU of a tile (coding_tree.cpp:628)
 * and does initialise them after PCM samples (coding_tree.cpp:1466); a PCM CU takes the QpY
 * of the CU before it (coding_tree.cpp:872) rather than qPY_PRED + CuQpDeltaVal. */
#define HEVCGEN_QUIRK_TILES_PCM  1
/* Dependent slice segments (not with WPP): the reference takes availability, the SAO merge
 * candidates and qPY_PREV per slice segment rather than per slice (coding_tree.cpp:189, :68,
 * :587), and its header parse of a dependent segment stops at slice_segment_address: no
 * entry points, and byte_alignment() only when the header is not byte aligned
 * (slice_header.cpp:141, decoder.cpp:243). */
#define HEVCGEN_QUIRK_DEPENDENT  2

void hevcgen_default_cfg(hevcgen_cfg_t* cfg, int32_t width, int32_t height, uint64_t seed);

/* The stream and, per picture, the records the generator drew: the TUs in decode order
 * (every TU of an intra CU; the coded ones of an inter CU, as a decoder dequantises them),
 * each coded one with its N x N levels at coeff_offset in the picture's level pool; and
 * the PUs in decode order: position and size, and for a PU coded with AMVP its ref_idx
 * (-1: list unused) and its coded mvd in mv (the decoder adds its predictor); a merged or
 * skipped PU has ref_idx -2 in both lists (the decoder derives its motion). */
typedef struct hevcgen_stream {
    uint8_t*  bytes;
    size_t    size;
    int32_t   pictures;
    int32_t*  num_tus;           /* per picture                                           */
    hevc_tu_t** tus;             /* per picture                                           */
    uint64_t* num_coeffs;        /* per picture                                           */
    int16_t** coeffs;            /* per picture                                           */
    int32_t*  slice_type;        /* per picture: 0 B, 1 P, 2 I (slice_type of 7.4.7.1)   */
    int32_t*  poc;               /* per picture: PicOrderCntVal (output order)            */
    int32_t*  output;            /* per picture: pic_output_flag                          */
    int32_t*  tid;               /* per picture: TemporalId                               */
    int32_t   crop[4];           /* conformance window: left, right, top, bottom, in      */
                                 /* chroma samples (SubWidthC = SubHeightC = 2)           */
    int32_t*  num_pus;           /* per picture                                           */
    hevc_pu_t** pus;             /* per picture                                           */
} hevcgen_stream_t;

hevcgen_stream_t* hevcgen_stream(const hevcgen_cfg_t* cfg);
void hevcgen_stream_free(hevcgen_stream_t* s);

#ifdef __cplusplus
}
#endif

#endif /* HEVC_BITGEN_H */
