/*
 * synth.h — seeded generator of reconstruction workloads (host only).
 *
 * It draws legal-shaped picture syntax (CTU quadtrees, CU prediction modes, PU
 * partitions and motion, transform trees with coefficient levels, intra modes, QPs,
 * SAO parameters) and derives the per-4x4 deblocking side information exactly the
 * way the hevc.js coding tree records it (src/decoding/coding_tree.cpp:960-1021 for
 * CU/PU edges, :1229-1248 for TU edges, src/decoding/decoder.cpp:140-147 for the
 * per-picture initial fill).  The same generated syntax drives the GPU back end, the
 * CPU restatement and the reference harness, so every arm sees identical inputs.
 *
 * Random numbers: std::mt19937_64 (its sequence is fixed by the C++ standard) mapped
 * to ranges by the helpers in synth.cpp; real-valued draws use 53-bit doubles.
 */
#ifndef HEVCSYNTH_H
#define HEVCSYNTH_H

#include "../../include/hevcgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hevcsynth_cfg {
    int32_t  width, height;      /* luma, multiples of 8                                */
    uint64_t seed;
    double   p_split;            /* CU quadtree split probability (down to 8x8)         */
    double   p_intra;            /* probability that a CU is intra                      */
    double   p_intra_nxn;        /* probability that an 8x8 intra CU is NxN             */
    double   p_skip;             /* probability that an inter CU is skipped             */
    double   p_bi;               /* probability that a PU is bi-predicted               */
    double   p_wp;               /* probability that a PU uses explicit WP              */
    double   p_merge;            /* probability that a PU copies the previous motion    */
    int32_t  mv_range;           /* MV components uniform in [-mv_range, mv_range] qpel */
    double   p_tu_split;         /* transform-tree split probability                    */
    double   p_cbf_luma;         /* cbf_luma probability per luma TU                    */
    double   p_cbf_chroma;       /* cbf_cb / cbf_cr probability per chroma node         */
    int32_t  qp_min, qp_max;     /* per-CU QpY range                                    */
    int32_t  sao;                /* draw SAO parameters per CTU                         */
    int32_t  num_refs;           /* reference pictures (1..2)                           */
    int32_t  slice_type;         /* 0 B, 1 P, 2 I                                       */
    int32_t  poc;                /* POC of the picture                                  */
    int32_t  strong_intra_smoothing;
    int32_t  cb_qp_offset, cr_qp_offset;
    int32_t  beta_offset_div2, tc_offset_div2;
    int32_t  scaling_lists;      /* attach scaling lists drawn by hevcsynth_scaling     */
    int32_t  log2_ctb;           /* CtbLog2SizeY 4..6; 0 means 6                        */
    int32_t  tile_cols, tile_rows;   /* uniformly spaced tiles (0 or 1: none); CTBs are  */
                                     /* then drawn in tile scan, the decoding order      */
    int32_t  no_lf_across_tiles; /* loop_filter_across_tiles_enabled_flag = 0           */
    double   p_pcm;              /* probability that a 2Nx2N intra CU of 8..32 is PCM   */
} hevcsynth_cfg_t;

/* One coding unit (synth-only: used by the reference harness to replay decode order). */
typedef struct hevcsynth_cu {
    uint16_t x, y;
    uint8_t  log2_size;
    uint8_t  pred_mode;          /* 0 inter, 1 intra, 2 skip (PredMode of types.h)      */
    uint8_t  part_mode;          /* PartMode of src/common/types.h                      */
    int8_t   qp_y;
    int32_t  first_pu, num_pu;
    int32_t  first_tu, num_tu;
    int32_t  has_tree;           /* transform tree present (not skip, rqt_root_cbf)    */
    int32_t  reserved;
} hevcsynth_cu_t;

typedef struct hevcsynth_picture {
    hevc_picture_syntax_t syn;   /* views into the arrays owned by this object          */
    int32_t               num_cus;
    const hevcsynth_cu_t* cus;
    void*                 impl;
} hevcsynth_picture_t;

/* Defaults of the reconstruction configs (CU split 0.5, QP 22..37, MV +-256 qpel, ...). */
void hevcsynth_default_cfg(hevcsynth_cfg_t* cfg, int32_t width, int32_t height, uint64_t seed);
/* Draw one picture of syntax.  Returns NULL on bad arguments. */
hevcsynth_picture_t* hevcsynth_picture(const hevcsynth_cfg_t* cfg);
void hevcsynth_picture_free(hevcsynth_picture_t* pic);

/* Picture content: each plane = 128 + sum of 8 2-D sinusoids (periods 8..256 px)
 * + uniform [-8, 8] noise, clipped to 0..255.  out is I420 (W*H*3/2 bytes). */
int hevcsynth_content(int32_t width, int32_t height, uint64_t seed, uint8_t* out);

/* Independent residual blocks: size mix DST4 25 %, DCT4 25 %, DCT8 25 %, DCT16 15 %,
 * DCT32 10 %, QP uniform in [qp_min, qp_max], levels nonzero with probability
 * 0.6*exp(-0.25*(u+v)), magnitude geometric(0.5), uniform sign; prediction uniform
 * 0..255.  Returns the number of coefficient slots (sum of N*N) or -1.
 * Call with NULL arrays to size them first. */
int64_t hevcsynth_blocks(int32_t num_tus, uint64_t seed, int32_t qp_min, int32_t qp_max,
                         hevc_tu_t* tus, int16_t* coeffs, uint8_t* pred);

/* Scaling lists for the dequantisation checks: per (sizeId, matrixId) a flat list of 16,
 * a ramp 16 + k*(u+v) (k uniform 0..12) or bytes uniform in 0..255 (a parsed list can
 * hold any byte, 0 included); DC values uniform in 0..255, 0 with probability 1/4. */
int hevcsynth_scaling(uint64_t seed, hevc_scaling_t* out);

/* Histogram of the boundary strengths that the deblocking filter will derive for a
 * picture (edges on the 8x8 grid, per 4-sample segment, picture-edge and disabled
 * edges excluded): counts[0..2] for Bs 0, 1, 2. */
int hevcsynth_bs_histogram(const hevc_picture_syntax_t* syn, int64_t counts[3]);

#ifdef __cplusplus
}
#endif

#endif
