/* bitgen.h — seeded generator of random-syntax HEVC Main-profile bitstreams.
 *
 * It draws a legal coding tree per CTU (CU splits, intra 2Nx2N / NxN partitions, intra
 * prediction modes, transform trees, coded blocks and their levels, SAO parameters, slice
 * QPs) and CABAC-encodes it (Rec. ITU-T H.265 clause 9.3: binarisations, context selection
 * and initialisation, arithmetic encoding) into an Annex-B byte stream of IDR pictures:
 * VPS, SPS, PPS, then one slice per picture.  The reference decoder parses these streams
 * (src/decoding/syntax_elements.cpp, residual_coding.cpp:175, cabac.cpp:38); the records
 * it produces are the ones the generator drew, which tests/test_bitgen.py checks.
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
} hevcgen_cfg_t;

void hevcgen_default_cfg(hevcgen_cfg_t* cfg, int32_t width, int32_t height, uint64_t seed);

/* The stream and, per picture, the TU records the generator drew (intra TUs in decode
 * order, each with its N x N levels at coeff_offset in the picture's level pool). */
typedef struct hevcgen_stream {
    uint8_t*  bytes;
    size_t    size;
    int32_t   pictures;
    int32_t*  num_tus;           /* per picture                                           */
    hevc_tu_t** tus;             /* per picture                                           */
    uint64_t* num_coeffs;        /* per picture                                           */
    int16_t** coeffs;            /* per picture                                           */
} hevcgen_stream_t;

hevcgen_stream_t* hevcgen_stream(const hevcgen_cfg_t* cfg);
void hevcgen_stream_free(hevcgen_stream_t* s);

#ifdef __cplusplus
}
#endif

#endif /* HEVC_BITGEN_H */
