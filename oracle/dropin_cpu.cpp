// dropin_cpu.cpp — TEST INFRASTRUCTURE ONLY: a CPU model of the part of the hevcgpu.h
// job ABI that the drop-in decoder (hevc.js_b200/dropin) calls, over the oracle's
// restatement (hevc_oracle.c).
//
// oracle/Makefile links it, instead of libhevcgpu.so, with the drop-in's own hooks.cpp and
// hevc_api.cpp and the reference's parser objects into _ref/libhevcdec_oracle.so.  That
// library decodes a stream exactly as libhevcdec_gpu.so does, except that each picture's
// records are reconstructed by the oracle: the tests run it on the CPU to check the
// drop-in's recording, slot and write-back logic against the reference's whole-file MD5s
// before (and independently of) the GPU.  Nothing in the product links it.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../include/hevcgpu.h"

extern "C" int oracle_reconstruct_picture(const hevc_picture_syntax_t* syn, const uint8_t* const* refs,
                                          int32_t num_refs, uint8_t* out);

struct hevcgpu_ctx {
    uint64_t launches = 0;
};
struct hevcgpu_stream {
    hevcgpu_ctx* ctx;
    int W, H;
    std::vector<std::vector<uint8_t>> slots;   // packed I420
};
struct hevcgpu_job {
    hevcgpu_stream* st;
    const hevc_picture_syntax_t* syn;   // the caller keeps the records until job_free
};

namespace {
thread_local std::string g_err;
int fail(int code, const char* fmt, ...) {
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}
}  // namespace

extern "C" {

const char* hevcgpu_last_error(void) { return g_err.c_str(); }

int hevcgpu_create(int device, hevcgpu_ctx_t** out) {
    (void)device;
    *out = new hevcgpu_ctx();
    return HEVCGPU_OK;
}

void hevcgpu_destroy(hevcgpu_ctx_t* ctx) { delete ctx; }

uint64_t hevcgpu_launch_count(hevcgpu_ctx_t* ctx) { return ctx ? ctx->launches : 0; }

int hevcgpu_stream_open(hevcgpu_ctx_t* ctx, int32_t width, int32_t height, int32_t bit_depth, int32_t num_slots,
                        hevcgpu_stream_t** out) {
    if (bit_depth != 8) return fail(HEVCGPU_EUNSUPPORTED, "bit depth %d", bit_depth);
    auto* st = new hevcgpu_stream{ctx, width, height, {}};
    st->slots.assign((size_t)num_slots, std::vector<uint8_t>((size_t)width * height * 3 / 2, 0));
    *out = st;
    return HEVCGPU_OK;
}

void hevcgpu_stream_close(hevcgpu_stream_t* st) { delete st; }

int hevcgpu_stream_sync(hevcgpu_stream_t* st) { return st ? HEVCGPU_OK : HEVCGPU_EINVAL; }

int hevcgpu_job_prepare(hevcgpu_stream_t* st, const hevc_picture_syntax_t* syn, hevcgpu_job_t** out) {
    if (syn->params.width != st->W || syn->params.height != st->H)
        return fail(HEVCGPU_EINVAL, "picture %dx%d on a %dx%d stream", syn->params.width, syn->params.height, st->W,
                    st->H);
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < syn->params.num_ref[l]; i++)
            if (syn->params.ref_slot[l][i] < 0 || syn->params.ref_slot[l][i] >= (int)st->slots.size())
                return fail(HEVCGPU_EINVAL, "reference list %d entry %d names slot %d", l, i, syn->params.ref_slot[l][i]);
    *out = new hevcgpu_job{st, syn};
    return HEVCGPU_OK;
}

void hevcgpu_job_free(hevcgpu_job_t* job) { delete job; }

int hevcgpu_job_launch(hevcgpu_job_t* job, int32_t dst_slot) {
    hevcgpu_stream* st = job->st;
    if (dst_slot < 0 || dst_slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", dst_slot);
    std::vector<const uint8_t*> refs(st->slots.size());
    for (size_t k = 0; k < st->slots.size(); k++) refs[k] = st->slots[k].data();
    std::vector<uint8_t> out(st->slots[(size_t)dst_slot].size());
    if (oracle_reconstruct_picture(job->syn, refs.data(), (int32_t)refs.size(), out.data()) != 0)
        return fail(HEVCGPU_EINVAL, "the oracle refused the records");
    st->slots[(size_t)dst_slot].swap(out);
    st->ctx->launches++;
    return HEVCGPU_OK;
}

int hevcgpu_slot_upload(hevcgpu_stream_t* st, int32_t slot, const uint8_t* i420) {
    if (!st || slot < 0 || slot >= (int)st->slots.size() || !i420) return fail(HEVCGPU_EINVAL, "bad slot %d", slot);
    st->slots[(size_t)slot].assign(i420, i420 + (size_t)st->W * st->H * 3 / 2);
    return HEVCGPU_OK;
}

int hevcgpu_slot_download_frame(hevcgpu_stream_t* st, int32_t slot, const hevc_crop_t* crop, uint16_t* y,
                                int32_t stride_y, uint16_t* cb, uint16_t* cr, int32_t stride_c) {
    if (slot < 0 || slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", slot);
    const hevc_crop_t c = crop ? *crop : hevc_crop_t{0, 0, 0, 0};
    const uint8_t* s = st->slots[(size_t)slot].data();
    const int W = st->W, H = st->H, w = W - c.left - c.right, h = H - c.top - c.bottom;
    uint16_t* dst[3] = {y, cb, cr};
    const int stride[3] = {stride_y, stride_c, stride_c};
    for (int p = 0; p < 3; p++) {
        const int pw = p ? W / 2 : W, ph = p ? H / 2 : H, sub = p ? 2 : 1;
        const uint8_t* plane = s + (p == 0 ? 0 : (size_t)W * H + (size_t)(p - 1) * (W / 2) * (H / 2));
        for (int yy = 0; yy < h / sub; yy++)
            for (int xx = 0; xx < w / sub; xx++)
                dst[p][(size_t)yy * stride[p] + xx] = plane[(size_t)(yy + c.top / sub) * pw + xx + c.left / sub];
        (void)ph;
    }
    return HEVCGPU_OK;
}

}  // extern "C"
