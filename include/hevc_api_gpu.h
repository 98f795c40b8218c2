/*
 * hevc_api_gpu.h — the hevc.js decoder's C API with reconstruction on the GPU.
 *
 * libhevcdec_gpu.so exports the same functions, with the same arguments, return codes,
 * ownership and threading rules, as privaloops/hevc.js src/wasm/hevc_api.h:13-86, so a
 * caller of the reference (its WASM/TypeScript binding, its CLI, its tests) links against
 * it unchanged.  Inside, the reference's own host decoder parses: NAL units, parameter
 * sets, slice headers, the DPB's POC/RPS/reference-list logic and CABAC (src/bitstream,
 * src/syntax, src/decoding) are compiled from the reference's sources.  Its six
 * reconstruction hooks (perform_dequant, perform_transform_inverse,
 * perform_intra_prediction, perform_inter_prediction, apply_deblocking, apply_sao) are
 * NOT linked: this library defines them, and they only record the picture's syntax as the
 * records of hevcgpu.h.  At the end of each picture the records go to the GPU (hevcgpu.h
 * job API, DPB slots in HBM) and the reconstructed picture is written back into the
 * reference's Picture planes, from which the frame calls below hand it out.  There is no
 * CPU reconstruction anywhere in the library.
 *
 * Layouts: HEVCFrame and HEVCStreamInfo are the reference's (hevc_api.h:21-42), field for
 * field, so that existing bindings read them unchanged.
 */
#ifndef HEVC_API_GPU_H
#define HEVC_API_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct HEVCDecoder HEVCDecoder;

/* A decoded frame: 16-bit planes inside the conformance window, in decoder-owned memory
 * valid until the next decode/feed/drain/flush call or destroy (hevc_api.h:21-33). */
typedef struct {
    const uint16_t* y;
    const uint16_t* cb;
    const uint16_t* cr;
    int width;
    int height;
    int stride_y;
    int stride_c;
    int chroma_width;
    int chroma_height;
    int bit_depth;
    int poc;
} HEVCFrame;

/* hevc_api.h:35-42 */
typedef struct {
    int width;
    int height;
    int bit_depth;
    int chroma_format;
    int profile;
    int level;
} HEVCStreamInfo;

#define HEVC_OK         0
#define HEVC_ERROR     -1
#define HEVC_NEED_MORE -2

/* hevc_api.h:46 / hevc_api.cpp:19.  Allocates host state only; the GPU context is made
 * at the first picture (device 0, or the device set by hevc_decoder_set_device). */
HEVCDecoder* hevc_decoder_create(void);
/* hevc_api.h:49 / hevc_api.cpp:23.  Waits for the decoder's GPU work, frees its slots. */
void hevc_decoder_destroy(HEVCDecoder* dec);
/* hevc_api.h:53 / hevc_api.cpp:27.  Parses every picture on the host and reconstructs
 * each on the GPU as soon as it is parsed (the next picture's parsing overlaps it);
 * returns once every picture's samples are in host memory.  HEVC_ERROR when the GPU
 * path fails or refuses a picture (hevc_decoder_last_error says why); a parse error after
 * some pictures hands out the pictures reconstructed before it, as the reference does. */
int hevc_decoder_decode(HEVCDecoder* dec, const uint8_t* data, size_t size);
/* hevc_api.h:56 / hevc_api.cpp:45 */
int hevc_decoder_get_frame_count(HEVCDecoder* dec);
/* hevc_api.h:61 / hevc_api.cpp:50.  Frames in (CVS, POC) order. */
int hevc_decoder_get_frame(HEVCDecoder* dec, int index, HEVCFrame* frame);
/* hevc_api.h:65 / hevc_api.cpp:176 */
int hevc_decoder_get_info(HEVCDecoder* dec, HEVCStreamInfo* info);
/* hevc_api.h:72 / hevc_api.cpp:85.  Complete NAL units; pictures are reconstructed as in
 * hevc_decoder_decode. */
int hevc_decoder_feed(HEVCDecoder* dec, const uint8_t* data, size_t size);
/* hevc_api.h:77 / hevc_api.cpp:96.  The reference's bumping process (dpb.cpp:459-506)
 * picks the pictures; the call returns once their samples are in host memory. */
int hevc_decoder_drain(HEVCDecoder* dec, int* count);
/* hevc_api.h:80 / hevc_api.cpp:109 */
int hevc_decoder_get_drained_frame(HEVCDecoder* dec, int index, HEVCFrame* frame);
/* hevc_api.h:84 / hevc_api.cpp:164 */
int hevc_decoder_flush(HEVCDecoder* dec);

/* ---- additions (no counterpart in the reference API) ---- */

/* Text of the decoder's last GPU-side failure ("" when none). */
const char* hevc_decoder_last_error(HEVCDecoder* dec);
/* CUDA device for the decoder's GPU context; only before its first picture. */
int hevc_decoder_set_device(HEVCDecoder* dec, int device);
/* Pictures reconstructed on the GPU by this decoder, and the kernel launches they took. */
int hevc_decoder_gpu_stats(HEVCDecoder* dec, uint64_t* pictures, uint64_t* launches);
/* Nanoseconds the decoder's calls have waited for the GPU back end so far (for room in its
 * queue of pictures, or for frames to be written back).  The rest of their time is the
 * host's own: NAL and slice parsing, CABAC and the recording of the picture's syntax. */
int hevc_decoder_gpu_wait_ns(HEVCDecoder* dec, uint64_t* ns);

#ifdef __cplusplus
}
#endif

#endif /* HEVC_API_GPU_H */
