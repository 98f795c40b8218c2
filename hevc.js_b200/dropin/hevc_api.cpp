// hevc_api.cpp — the hevc.js decoder C API (include/hevc_api_gpu.h) over the reference's
// host decoder with reconstruction on the GPU.
//
// Same functions, arguments, return codes and ownership as privaloops/hevc.js
// src/wasm/hevc_api.cpp:9-189.  The decoder is the reference's hevc::Decoder; its
// reconstruction hooks are the recording ones of hooks.cpp, so every picture it parses is
// reconstructed by the GPU back end, one picture behind the parser, and written back into
// the Picture the reference hands out.  Each call that hands out frames first waits until
// the GPU has written them.  Frames the GPU did not reconstruct (a picture cut short by a
// parse error) are not handed out.
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "backend.h"
#include "decoding/decoder.h"

#include "hevc_api_gpu.h"

struct HEVCDecoder {
    hevc::Decoder decoder;
    dropin::Backend* gpu = nullptr;
    std::vector<hevc::Picture*> output;    // batch mode
    std::vector<hevc::Picture*> drained;   // incremental mode
    ~HEVCDecoder() { dropin::detach(gpu); }
};

namespace {

// Only pictures whose samples the GPU wrote back.
std::vector<hevc::Picture*> written(HEVCDecoder* dec, const std::vector<hevc::Picture*>& pics) {
    std::vector<hevc::Picture*> out;
    out.reserve(pics.size());
    for (hevc::Picture* p : pics)
        if (dropin::reconstructed(dec->gpu, p)) out.push_back(p);
    return out;
}

void fill(const hevc::Picture* pic, HEVCFrame* frame) {
    const int sub_w = hevc::SubWidthC(pic->chroma_format), sub_h = hevc::SubHeightC(pic->chroma_format);
    const int crop_w = pic->pic_width_in_luma - pic->conf_win_left - pic->conf_win_right;
    const int crop_h = pic->pic_height_in_luma - pic->conf_win_top - pic->conf_win_bottom;
    const int y_off = pic->conf_win_top * pic->stride[0] + pic->conf_win_left;
    const int c_off = (pic->conf_win_top / sub_h) * pic->stride[1] + pic->conf_win_left / sub_w;
    frame->y = pic->planes[0].data() + y_off;
    frame->cb = pic->planes[1].data() + c_off;
    frame->cr = pic->planes[2].data() + c_off;
    frame->width = crop_w;
    frame->height = crop_h;
    frame->stride_y = pic->stride[0];
    frame->stride_c = pic->stride[1];
    frame->chroma_width = crop_w / sub_w;
    frame->chroma_height = crop_h / sub_h;
    frame->bit_depth = pic->bit_depth_luma;
    frame->poc = pic->poc;
}

}  // namespace

extern "C" {

HEVCDecoder* hevc_decoder_create(void) {
    HEVCDecoder* dec = new (std::nothrow) HEVCDecoder();
    if (!dec) return nullptr;
    dec->gpu = dropin::attach(&dec->decoder.dpb(), true);
    return dec;
}

void hevc_decoder_destroy(HEVCDecoder* dec) { delete dec; }

int hevc_decoder_decode(HEVCDecoder* dec, const uint8_t* data, size_t size) {
    if (!dec || !data || size == 0) return HEVC_ERROR;
    hevc::DecodeStatus status = hevc::DecodeStatus::OK;
    bool threw = false;
    try {
        status = dec->decoder.decode(data, size);
    } catch (...) {
        threw = true;   // as the reference: hand out what was decoded before the exception
    }
    if (dropin::finish(dec->gpu) != 0) {
        dec->output.clear();
        return HEVC_ERROR;
    }
    if (!threw && status != hevc::DecodeStatus::OK) return HEVC_ERROR;
    dec->output = written(dec, dec->decoder.output_pictures());
    if (threw) return dec->output.empty() ? HEVC_ERROR : HEVC_OK;
    return HEVC_OK;
}

int hevc_decoder_get_frame_count(HEVCDecoder* dec) { return dec ? (int)dec->output.size() : 0; }

int hevc_decoder_get_frame(HEVCDecoder* dec, int index, HEVCFrame* frame) {
    if (!dec || !frame || index < 0 || index >= (int)dec->output.size()) return HEVC_ERROR;
    fill(dec->output[(size_t)index], frame);
    return HEVC_OK;
}

int hevc_decoder_feed(HEVCDecoder* dec, const uint8_t* data, size_t size) {
    if (!dec || !data || size == 0) return HEVC_ERROR;
    hevc::DecodeStatus s;
    try {
        s = dec->decoder.feed(data, size);
    } catch (...) {
        dropin::finish(dec->gpu);
        return HEVC_ERROR;
    }
    if (dropin::finish(dec->gpu) != 0) return HEVC_ERROR;
    return s == hevc::DecodeStatus::OK ? HEVC_OK : HEVC_ERROR;
}

int hevc_decoder_drain(HEVCDecoder* dec, int* count) {
    if (!dec || !count) return HEVC_ERROR;
    try {
        if (dropin::finish(dec->gpu) != 0) {
            *count = 0;
            return HEVC_ERROR;
        }
        dec->drained = written(dec, dec->decoder.drain());
        *count = (int)dec->drained.size();
        return HEVC_OK;
    } catch (...) {
        *count = 0;
        return HEVC_ERROR;
    }
}

int hevc_decoder_get_drained_frame(HEVCDecoder* dec, int index, HEVCFrame* frame) {
    if (!dec || !frame || index < 0 || index >= (int)dec->drained.size()) return HEVC_ERROR;
    fill(dec->drained[(size_t)index], frame);
    return HEVC_OK;
}

int hevc_decoder_flush(HEVCDecoder* dec) {
    if (!dec) return HEVC_ERROR;
    try {
        if (dropin::finish(dec->gpu) != 0) return HEVC_ERROR;
        dec->drained = written(dec, dec->decoder.flush());
        return HEVC_OK;
    } catch (...) {
        return HEVC_ERROR;
    }
}

int hevc_decoder_get_info(HEVCDecoder* dec, HEVCStreamInfo* info) {
    if (!dec || !info || dec->output.empty()) return HEVC_ERROR;
    const hevc::Picture* pic = dec->output[0];
    info->width = pic->pic_width_in_luma - pic->conf_win_left - pic->conf_win_right;
    info->height = pic->pic_height_in_luma - pic->conf_win_top - pic->conf_win_bottom;
    info->bit_depth = pic->bit_depth_luma;
    info->chroma_format = static_cast<int>(pic->chroma_format);
    info->profile = 0;
    info->level = 0;
    return HEVC_OK;
}

const char* hevc_decoder_last_error(HEVCDecoder* dec) { return dec ? dropin::last_error(dec->gpu) : "null decoder"; }

int hevc_decoder_set_device(HEVCDecoder* dec, int device) {
    return dec && dropin::set_device(dec->gpu, device) == 0 ? HEVC_OK : HEVC_ERROR;
}

int hevc_decoder_gpu_stats(HEVCDecoder* dec, uint64_t* pictures, uint64_t* launches) {
    if (!dec) return HEVC_ERROR;
    dropin::stats(dec->gpu, pictures, launches);
    return HEVC_OK;
}

int hevc_decoder_gpu_wait_ns(HEVCDecoder* dec, uint64_t* ns) {
    if (!dec || !ns) return HEVC_ERROR;
    *ns = dropin::wait_ns(dec->gpu);
    return HEVC_OK;
}

}  // extern "C"
