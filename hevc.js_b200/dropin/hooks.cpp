// hooks.cpp — the reconstruction hooks of privaloops/hevc.js's decoder, defined so that
// they only record, and the GPU back end the records go to.
//
// The reference's coding tree (src/decoding/coding_tree.cpp, compiled from its sources
// into this library) calls six functions for the samples of a picture:
//   perform_dequant            src/decoding/transform.cpp:293
//   perform_transform_inverse  src/decoding/transform.cpp:374
//   perform_intra_prediction   src/decoding/intra_prediction.cpp:428
//   perform_inter_prediction   src/decoding/interpolation.cpp:306
//   apply_deblocking           src/filters/deblocking.cpp:357
//   apply_sao                  src/filters/sao.cpp:20
// The objects that define them in the reference are not linked into this library: the
// definitions below are the only ones.  They write no sample.  The first four record the
// picture's transform and prediction units as the TU/PU records of hevcgpu.h;
// apply_deblocking reads the DecodingContext's grids (CUInfo, the 4x4 edge/cbf/TU-size
// maps, SAO parameters, slice and tile ids, scaling lists, the DPB's reference lists) into
// the remaining records, the state the reference's filters read (decoder.cpp:117-185
// fills it); apply_sao sends the picture to the GPU: a job into a DPB slot in HBM whose
// reference slots are the slots of the pictures in the reference lists, then the
// reconstructed picture back into the reference's Picture planes (16-bit, full picture).
//
// Levels are taken where the residual syntax produces them: decode_residual_coding
// (src/decoding/residual_coding.cpp:175) is wrapped at link time (-Wl,--wrap), so that
// transquant-bypass TUs, whose levels the coding tree copies without calling any hook
// (coding_tree.cpp:1302-1304), are recorded too.  PCM samples are written by the parser
// straight into the Picture (coding_tree.cpp:1425-1469); apply_deblocking reads them back
// from there for the CUs the CUInfo grid marks as PCM.
//
// With WPP the coding tree runs CTU rows on the decoder's thread pool, so the hooks run on
// several threads: a TU's state between its levels and its prediction is per thread, and
// the picture's record arrays take a lock.  A CTU row starts only after the two CTUs above
// it are done, so records appended in call order are in a valid decode order for the
// GPU's intra schedule (each TU after every TU whose samples it reads).
#include "backend.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common/picture.h"
#include "common/types.h"
#include "decoding/coding_tree.h"
#include "decoding/dpb.h"
#include "syntax/pps.h"
#include "syntax/slice_header.h"
#include "syntax/sps.h"

#include "hevcgpu.h"

using hevc::DecodingContext;
using hevc::Picture;

namespace dropin {

// One parsed picture on its way to the GPU: its records and the Picture its samples go to
// (held, so that the DPB's eviction cannot free the planes before the write-back).
struct Work {
    std::shared_ptr<Picture> pic;
    int slot = -1;
    int fill_generated = -1;   // a slot to fill with the generated picture before this one
    hevc_picture_syntax_t syn{};
    std::vector<hevc_tu_t> tus;
    std::vector<int16_t> coeffs;
    std::vector<hevc_pu_t> pus;
    std::vector<hevc_wp_t> wp;
    std::vector<const Picture*> pu_ref[2];   // per PU: the picture each used list points at
    std::vector<uint32_t> blk;
    std::vector<hevc_sao_t> sao;
    std::vector<uint8_t> ctb_slice;
    std::vector<uint16_t> ctb_tile;
    std::vector<hevc_slice_t> slices;
    hevc_scaling_t scaling{};
    bool has_scaling = false, has_tiles = false;
    std::string unsupported;

    void clear() {
        tus.clear();
        coeffs.clear();
        pus.clear();
        wp.clear();
        pu_ref[0].clear();
        pu_ref[1].clear();
        unsupported.clear();
        pic.reset();
        slot = -1;
        fill_generated = -1;
    }
};

class Backend {
public:
    const hevc::DPB* dpb = nullptr;
    bool deferred = false;
    int device = 0;

    // ---- recording (parse thread and WPP workers) ----
    std::mutex rec_mu;
    std::unique_ptr<Work> cur{new Work()};

    // ---- GPU state (parse thread; the worker only runs jobs) ----
    hevcgpu_ctx_t* gctx = nullptr;
    hevcgpu_stream_t* st = nullptr;
    int W = 0, H = 0;
    struct Slot {
        std::weak_ptr<Picture> pic;
        const Picture* raw = nullptr;
        bool used = false;
        bool generated = false;   // holds the generated picture of 8.3.3.2, not a decoded one
    };
    std::vector<Slot> slots;
    int gen_slot = -1;                // the slot with the generated picture, once one was needed
    std::vector<uint8_t> gen_samples; // its I420 samples (1 << (BitDepth - 1) everywhere)

    // ---- worker (deferred mode) ----
    std::mutex q_mu;
    std::condition_variable q_cv, idle_cv;
    std::deque<std::unique_ptr<Work>> queue;
    std::vector<std::unique_ptr<Work>> spare;   // recycled record buffers
    bool busy = false, stop = false;
    std::thread worker;
    std::string error;   // first failure; guarded by q_mu
    std::map<const Picture*, std::weak_ptr<Picture>> done;   // written back; guarded by q_mu
    uint64_t pictures = 0;
    uint64_t wait_ns = 0;   // guarded by q_mu

    ~Backend() {
        {
            std::lock_guard<std::mutex> g(q_mu);
            stop = true;
        }
        q_cv.notify_all();
        if (worker.joinable()) worker.join();
        if (st) hevcgpu_stream_close(st);
        if (gctx) hevcgpu_destroy(gctx);
    }

    void fail(const std::string& why) {
        std::lock_guard<std::mutex> g(q_mu);
        if (error.empty()) error = why;
    }
    std::string current_error() {
        std::lock_guard<std::mutex> g(q_mu);
        return error;
    }
    [[noreturn]] void raise() { throw std::runtime_error("hevc GPU back end: " + current_error()); }

    void note_unsupported(const std::string& why) {
        std::lock_guard<std::mutex> g(rec_mu);
        if (cur->unsupported.empty()) cur->unsupported = why;
    }

    void append_tu(hevc_tu_t t, const int16_t* lv, int n) {
        std::lock_guard<std::mutex> g(rec_mu);
        if (t.flags & HEVC_TU_CODED) {
            t.coeff_offset = (uint32_t)cur->coeffs.size();
            cur->coeffs.insert(cur->coeffs.end(), lv, lv + n);
        }
        cur->tus.push_back(t);
    }

    void finish_records(DecodingContext& ctx);
    void submit(DecodingContext& ctx);
    int run(Work& w);   // on the worker, or inline
    int wait_idle();
    void worker_loop();
    int ensure_gpu(const hevc::SPS& sps);
};

namespace {

std::mutex g_reg_mu;
std::unordered_map<const hevc::DPB*, Backend*> g_reg;
std::atomic<uint64_t> g_reg_gen{1};

struct Cached {
    const hevc::DPB* dpb = nullptr;
    Backend* b = nullptr;
    uint64_t gen = 0;
};
thread_local Cached t_cached;

Backend* lookup(const hevc::DPB* dpb) {
    const uint64_t gen = g_reg_gen.load(std::memory_order_acquire);
    if (t_cached.dpb == dpb && t_cached.gen == gen) return t_cached.b;
    Backend* b = attach(dpb, false);
    t_cached = Cached{dpb, b, gen};
    return b;
}

// A TU between its levels (decode_residual_coding) and the hook that completes it.
struct Pending {
    bool active = false;
    Backend* b = nullptr;   // the decoder of the TU
    hevc_tu_t t{};
    int16_t lv[32 * 32];
    int n = 0;
};
thread_local Pending t_pending;

}  // namespace

Backend* attach(const hevc::DPB* dpb, bool deferred) {
    std::lock_guard<std::mutex> g(g_reg_mu);
    auto it = g_reg.find(dpb);
    if (it != g_reg.end()) {
        if (deferred) it->second->deferred = true;
        return it->second;
    }
    Backend* b = new Backend();
    b->dpb = dpb;
    b->deferred = deferred;
    g_reg[dpb] = b;
    g_reg_gen.fetch_add(1, std::memory_order_release);
    return b;
}

void detach(Backend* b) {
    if (!b) return;
    {
        std::lock_guard<std::mutex> g(g_reg_mu);
        g_reg.erase(b->dpb);
        g_reg_gen.fetch_add(1, std::memory_order_release);
    }
    b->wait_idle();
    delete b;
}

int finish(Backend* b) { return b ? b->wait_idle() : -1; }

const char* last_error(Backend* b) {
    if (!b) return "no decoder";
    static thread_local std::string msg;
    msg = b->current_error();
    return msg.c_str();
}

int set_device(Backend* b, int device) {
    if (!b || b->gctx || device < 0) return -1;
    b->device = device;
    return 0;
}

bool reconstructed(Backend* b, const Picture* pic) {
    std::lock_guard<std::mutex> g(b->q_mu);
    auto it = b->done.find(pic);
    return it != b->done.end() && it->second.lock().get() == pic;
}

void stats(Backend* b, uint64_t* pictures, uint64_t* launches) {
    std::lock_guard<std::mutex> g(b->q_mu);
    if (pictures) *pictures = b->pictures;
    if (launches) *launches = b->gctx ? hevcgpu_launch_count(b->gctx) : 0;
}

int Backend::wait_idle() {
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_lock<std::mutex> g(q_mu);
    idle_cv.wait(g, [&] { return queue.empty() && !busy; });
    wait_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
    return error.empty() ? 0 : -1;
}

uint64_t wait_ns(Backend* b) {
    if (!b) return 0;
    std::lock_guard<std::mutex> g(b->q_mu);
    return b->wait_ns;
}

void Backend::worker_loop() {
    for (;;) {
        std::unique_ptr<Work> w;
        {
            std::unique_lock<std::mutex> g(q_mu);
            q_cv.wait(g, [&] { return stop || !queue.empty(); });
            if (queue.empty()) return;
            w = std::move(queue.front());
            queue.pop_front();
            busy = true;
        }
        const bool ok = error.empty() && run(*w) == 0;
        (void)ok;
        w->clear();
        {
            std::lock_guard<std::mutex> g(q_mu);
            spare.push_back(std::move(w));
            busy = false;
        }
        idle_cv.notify_all();
        q_cv.notify_all();
    }
}

// Prepare + launch the picture's job into its slot, then write the slot back into the
// Picture's planes (the call waits for the device).  Jobs run strictly one after another,
// so a slot reused by a later picture is written only after every earlier read of it.
int Backend::run(Work& w) {
    hevcgpu_job_t* job = nullptr;
    int rc = HEVCGPU_OK;
    if (w.fill_generated >= 0) {   // the generated picture, written before the first picture that reads it
        gen_samples.assign((size_t)W * H * 3 / 2, 128);
        rc = hevcgpu_slot_upload(st, w.fill_generated, gen_samples.data());
    }
    if (rc == HEVCGPU_OK) rc = hevcgpu_job_prepare(st, &w.syn, &job);
    if (rc == HEVCGPU_OK) rc = hevcgpu_job_launch(job, w.slot);
    Picture& p = *w.pic;
    if (rc == HEVCGPU_OK)
        rc = hevcgpu_slot_download_frame(st, w.slot, nullptr, p.planes[0].data(), p.stride[0], p.planes[1].data(),
                                         p.planes[2].data(), p.stride[1]);
    if (rc == HEVCGPU_OK) rc = hevcgpu_stream_sync(st);   // the device status of the launch
    const std::string msg = rc == HEVCGPU_OK ? std::string() : std::string(hevcgpu_last_error());
    if (job) hevcgpu_job_free(job);
    std::lock_guard<std::mutex> g(q_mu);
    if (rc != HEVCGPU_OK) {
        char buf[64];
        std::snprintf(buf, sizeof buf, "picture POC %d: ", p.poc);
        if (error.empty()) error = buf + msg;
        return -1;
    }
    done[w.pic.get()] = w.pic;
    pictures++;
    return 0;
}

int Backend::ensure_gpu(const hevc::SPS& sps) {
    const int w = (int)sps.pic_width_in_luma_samples, h = (int)sps.pic_height_in_luma_samples;
    if (!gctx) {
        if (hevcgpu_create(device, &gctx) != HEVCGPU_OK) {
            fail(std::string("no GPU context: ") + hevcgpu_last_error());
            return -1;
        }
    }
    if (st && w == W && h == H) return 0;
    if (wait_idle()) return -1;
    if (st) hevcgpu_stream_close(st);
    st = nullptr;
    slots.clear();
    gen_slot = -1;
    // every picture the DPB may hold as a reference, the current one, and two spare so that
    // the worker can still be writing back a picture whose slot is no longer a reference
    const int tid = (int)sps.sps_max_sub_layers_minus1;
    const int dpb_size = (int)sps.sub_layer_ordering[(size_t)tid].max_dec_pic_buffering_minus1 + 1;
    const int n = std::min(64, std::max(8, dpb_size + 3));
    if (hevcgpu_stream_open(gctx, w, h, 8, n, &st) != HEVCGPU_OK) {
        fail(std::string("stream: ") + hevcgpu_last_error());
        return -1;
    }
    W = w;
    H = h;
    slots.assign((size_t)n, Slot{});
    return 0;
}

// The records the reference's filters read from the DecodingContext, read at the point
// where they would run (deblocking.cpp:357, sao.cpp:20).
void Backend::finish_records(DecodingContext& ctx) {
    const hevc::SPS& sps = *ctx.sps;
    const hevc::PPS& pps = *ctx.pps;
    Work& w = *cur;
    const int Wp = (int)sps.pic_width_in_luma_samples, Hp = (int)sps.pic_height_in_luma_samples;
    const int gw = Wp / 4, gh = Hp / 4, nctb = (int)sps.PicSizeInCtbsY;
    if (sps.BitDepthY != 8 || sps.BitDepthC != 8)
        w.unsupported = "bit depth " + std::to_string(sps.BitDepthY) + " (the GPU path is 8-bit)";
    if (sps.chroma_format_idc != 1) w.unsupported = "chroma format other than 4:2:0";
    w.blk.resize((size_t)gw * gh);
    struct PcmCu {
        int x, y, log2;
    };
    std::vector<PcmCu> pcm;
    for (int gy = 0; gy < gh; gy++) {
        const size_t g0 = (size_t)gy * ctx.filter_grid_stride;
        for (int gx = 0; gx < gw; gx++) {
            const size_t g = g0 + gx;
            const hevc::CUInfo& cu = ctx.cu_at(gx * 4, gy * 4);
            uint32_t b = (ctx.edge_flags_v[g] ? HEVC_BLK_EDGE_V : 0u) | (ctx.edge_flags_h[g] ? HEVC_BLK_EDGE_H : 0u) |
                         (ctx.cbf_luma_grid[g] ? HEVC_BLK_CBF : 0u) |
                         (cu.pred_mode == hevc::PredMode::MODE_INTRA ? HEVC_BLK_INTRA : 0u) |
                         (cu.is_pcm ? HEVC_BLK_PCM : 0u) | (cu.cu_transquant_bypass ? HEVC_BLK_BYPASS : 0u) |
                         ((uint32_t)ctx.log2_tu_size_grid[g] << HEVC_BLK_TU_SHIFT) |
                         ((uint32_t)(uint8_t)cu.qp_y << HEVC_BLK_QP_SHIFT);
            w.blk[(size_t)gy * gw + gx] = b;
            // a PCM CU, once, at its top-left 4x4 unit
            if (cu.is_pcm) {
                const int x = gx * 4, y = gy * 4, s = 1 << cu.log2CbSize;
                if ((x & (s - 1)) == 0 && (y & (s - 1)) == 0) pcm.push_back({x, y, cu.log2CbSize});
            }
        }
    }
    // PCM CUs: the samples the parser stored in the Picture are the levels of PCM records
    // (HEVC_TU_PCM), inserted into decode order below.
    if (!pcm.empty()) {
        const Picture& pic = *ctx.pic;
        for (const PcmCu& c : pcm) {
            for (int ci = 0; ci < 3; ci++) {
                const int sub = ci ? 2 : 1, n = (1 << c.log2) / sub;
                hevc_tu_t t{};
                t.x = (uint16_t)(c.x / sub);
                t.y = (uint16_t)(c.y / sub);
                t.log2_size = (uint8_t)(c.log2 - (ci ? 1 : 0));
                t.c_idx = (uint8_t)ci;
                t.flags = HEVC_TU_INTRA | HEVC_TU_CODED | HEVC_TU_PCM;
                t.coeff_offset = (uint32_t)w.coeffs.size();
                for (int yy = 0; yy < n; yy++)
                    for (int xx = 0; xx < n; xx++)
                        w.coeffs.push_back((int16_t)pic.planes[ci][(size_t)(t.y + yy) * pic.stride[ci] + t.x + xx]);
                w.tus.push_back(t);
            }
        }
        // decode order: CTBs in tile scan, then z-order inside the CTB (a quadtree's
        // depth-first order is the Morton order of its blocks' corners); planes do not read
        // each other, so their relative order is free
        const int lc = (int)sps.CtbLog2SizeY, wctb = (int)sps.PicWidthInCtbsY;
        auto morton = [](uint32_t x, uint32_t y) {
            uint32_t m = 0;
            for (int i = 0; i < 8; i++) m |= ((x >> i) & 1u) << (2 * i) | ((y >> i) & 1u) << (2 * i + 1);
            return m;
        };
        std::vector<std::pair<uint64_t, uint32_t>> key(w.tus.size());
        for (size_t i = 0; i < w.tus.size(); i++) {
            const hevc_tu_t& t = w.tus[i];
            const int sub = t.c_idx ? 2 : 1, x = t.x * sub, y = t.y * sub;
            const int rs = (y >> lc) * wctb + (x >> lc);
            const uint64_t ts = pps.CtbAddrRsToTs.empty() ? (uint64_t)rs : (uint64_t)pps.CtbAddrRsToTs[(size_t)rs];
            const uint32_t z = morton((uint32_t)(x & ((1 << lc) - 1)) >> 2, (uint32_t)(y & ((1 << lc) - 1)) >> 2);
            key[i] = {(ts << 32) | ((uint64_t)z << 2) | t.c_idx, (uint32_t)i};
        }
        std::stable_sort(key.begin(), key.end(),
                         [](const std::pair<uint64_t, uint32_t>& a, const std::pair<uint64_t, uint32_t>& b) {
                             return a.first < b.first;
                         });
        std::vector<hevc_tu_t> sorted(w.tus.size());
        for (size_t i = 0; i < key.size(); i++) sorted[i] = w.tus[key[i].second];
        w.tus.swap(sorted);
    }
    w.sao.resize((size_t)nctb);
    for (int a = 0; a < nctb; a++) {
        const auto& s = ctx.sao_params[a];
        hevc_sao_t& o = w.sao[(size_t)a];
        for (int c = 0; c < 3; c++) {
            o.type[c] = (uint8_t)s.sao_type_idx[c];
            o.band_pos[c] = (uint8_t)s.sao_band_position[c];
            o.eo_class[c] = (uint8_t)s.sao_eo_class[c];
            for (int k = 0; k < 5; k++) o.offset[c][k] = (int8_t)s.sao_offset_val[c][k];
        }
    }
    w.ctb_slice.assign(ctx.slice_idx, ctx.slice_idx + nctb);
    w.slices.clear();
    for (int k = 0; k < ctx.num_slices; k++) {
        const hevc::SliceHeader& s = *ctx.slice_headers[k];
        w.slices.push_back(hevc_slice_t{(int8_t)s.slice_beta_offset_div2, (int8_t)s.slice_tc_offset_div2,
                                        (uint8_t)s.slice_deblocking_filter_disabled_flag,
                                        (uint8_t)s.slice_loop_filter_across_slices_enabled_flag});
    }
    w.has_tiles = !pps.TileId.empty() && !pps.CtbAddrRsToTs.empty();
    if (w.has_tiles) {
        w.ctb_tile.resize((size_t)nctb);
        for (int a = 0; a < nctb; a++) w.ctb_tile[(size_t)a] = (uint16_t)pps.TileId[(size_t)pps.CtbAddrRsToTs[(size_t)a]];
    }
    w.has_scaling = sps.scaling_list_enabled_flag;
    if (w.has_scaling) {
        const hevc::ScalingListData& sl =
            pps.pps_scaling_list_data_present_flag ? pps.scaling_list_data : sps.scaling_list_data;
        for (int sz = 0; sz < 4; sz++)
            for (int m = 0; m < 6; m++) std::memcpy(w.scaling.list[sz][m], sl.scaling_list[(size_t)sz][(size_t)m].data(), 64);
        for (int i = 0; i < 2; i++)
            for (int m = 0; m < 6; m++) w.scaling.dc[i][m] = sl.scaling_list_dc[(size_t)i][(size_t)m];
    }

    hevc_pic_params_t& p = w.syn.params;
    std::memset(&p, 0, sizeof(p));
    p.width = Wp;
    p.height = Hp;
    p.bit_depth = 8;
    p.log2_ctb = (int)sps.CtbLog2SizeY;
    p.log2_min_cb = (int)sps.log2_min_luma_coding_block_size_minus3 + 3;
    p.log2_min_tb = (int)sps.log2_min_luma_transform_block_size_minus2 + 2;
    p.strong_intra_smoothing = sps.strong_intra_smoothing_enabled_flag;
    p.intra_smoothing_disabled = sps.intra_smoothing_disabled_flag;
    p.pcm_loop_filter_disabled = sps.pcm_loop_filter_disabled_flag;
    p.sao_enabled = sps.sample_adaptive_offset_enabled_flag;
    p.cb_qp_offset = pps.pps_cb_qp_offset;
    p.cr_qp_offset = pps.pps_cr_qp_offset;
    p.tiles_enabled = pps.tiles_enabled_flag;
    p.loop_filter_across_tiles = pps.loop_filter_across_tiles_enabled_flag;
}

// Slots, reference slots and the hand-over of the picture to the GPU.
void Backend::submit(DecodingContext& ctx) {
    if (!current_error().empty()) raise();
    Work& w = *cur;
    if (!w.unsupported.empty()) {
        fail("picture POC " + std::to_string(ctx.pic->poc) + " is not supported: " + w.unsupported);
        raise();
    }
    // Every luma sample is predicted once: by the luma TUs of intra CUs (PCM included) and
    // by the PUs of inter CUs.  More than the picture's area means slices that code some
    // blocks twice (a damaged stream: the reference keeps whichever came last); the records
    // cannot say which, so the picture fails here rather than differ silently.
    {
        uint64_t area = 0;
        for (const hevc_tu_t& t : w.tus)
            if (t.c_idx == 0 && (t.flags & HEVC_TU_INTRA)) area += (uint64_t)1 << (2 * t.log2_size);
        for (const hevc_pu_t& u : w.pus) area += (uint64_t)u.w * u.h;
        const uint64_t pic_area = (uint64_t)ctx.sps->pic_width_in_luma_samples * ctx.sps->pic_height_in_luma_samples;
        if (area > pic_area) {
            fail("picture POC " + std::to_string(ctx.pic->poc) +
                 ": its slices code some blocks more than once (a damaged stream)");
            raise();
        }
    }
    if (ensure_gpu(*ctx.sps)) raise();
    const hevc::DPB& d = *ctx.dpb;
    // the shared pointer of the current picture, and the slots whose pictures are gone or
    // no longer references (the RPS of this picture has been applied)
    std::shared_ptr<Picture> self;
    for (const auto& sp : d.pictures())
        if (sp.get() == ctx.pic) self = sp;
    if (!self) {
        fail("the current picture is not in the DPB");
        raise();
    }
    for (Slot& s : slots) {
        if (!s.used || s.generated) continue;
        std::shared_ptr<Picture> p = s.pic.lock();
        if (!p || !p->is_reference()) s = Slot{};
    }
    int dst = -1;
    for (size_t k = 0; k < slots.size() && dst < 0; k++)
        if (!slots[k].used) dst = (int)k;
    if (dst < 0) {
        fail("no free DPB slot: more reference pictures than the stream's " + std::to_string(slots.size()) + " slots");
        raise();
    }
    auto slot_of = [&](const Picture* pic) {
        if (!pic) return -1;
        for (size_t k = 0; k < slots.size(); k++)
            if (slots[k].used && slots[k].raw == pic && slots[k].pic.lock().get() == pic) return (int)k;
        return -1;
    };
    hevc_pic_params_t& p = w.syn.params;
    const int n_list[2] = {d.num_ref_list0(), d.num_ref_list1()};
    const int other = dst == 0 ? 1 : 0;   // a valid slot for entries no PU uses
    int missing[2][16] = {};
    for (int l = 0; l < 2; l++) {
        p.num_ref[l] = std::min(n_list[l], 16);
        for (int i = 0; i < 16; i++) {
            p.ref_poc[l][i] = -999999;
            p.ref_slot[l][i] = -1;
        }
        for (int i = 0; i < p.num_ref[l]; i++) {
            const Picture* rp = l == 0 ? d.ref_pic_list0(i) : d.ref_pic_list1(i);
            const int s = slot_of(rp);
            if (rp) p.ref_poc[l][i] = rp->poc;
            p.ref_slot[l][i] = s >= 0 ? s : other;
            missing[l][i] = s < 0;
        }
    }
    // every PU must predict from the picture the final lists name at its index: the
    // records carry one pair of lists per picture, the pair the reference's deblocking
    // reads (deblocking.cpp:183-193)
    bool reads_missing = false;
    for (size_t k = 0; k < w.pus.size(); k++)
        for (int l = 0; l < 2; l++) {
            const int idx = w.pus[k].ref_idx[l];
            if (idx < 0) continue;
            const Picture* want = idx < p.num_ref[l] ? (l == 0 ? d.ref_pic_list0(idx) : d.ref_pic_list1(idx)) : nullptr;
            if (want != w.pu_ref[l][k]) {
                fail("picture POC " + std::to_string(ctx.pic->poc) +
                     ": slices with different reference lists are not supported");
                raise();
            }
            reads_missing = reads_missing || missing[l][idx];
        }
    // A list entry with no picture ("no reference picture": a RASL picture of the CRA picture
    // decoding started at, whose references precede it) is the generated picture of 8.3.3.2,
    // every sample 1 << (BitDepth - 1), in a slot kept for it.  (The reference predicts from
    // its uninitialised prediction buffer there, interpolation.cpp:327-331; the standard does
    // not output such a picture.)
    if (reads_missing) {
        if (gen_slot < 0) {
            for (size_t k = 0; k < slots.size() && gen_slot < 0; k++)
                if (!slots[k].used && (int)k != dst) gen_slot = (int)k;
            if (gen_slot < 0) {
                fail("no free DPB slot for the generated reference picture");
                raise();
            }
            slots[(size_t)gen_slot] = Slot{{}, nullptr, true, true};
            w.fill_generated = gen_slot;
        }
        for (int l = 0; l < 2; l++)
            for (int i = 0; i < p.num_ref[l]; i++)
                if (missing[l][i]) p.ref_slot[l][i] = gen_slot;
    }
    slots[(size_t)dst] = Slot{self, self.get(), true};
    w.pic = self;
    w.slot = dst;
    hevc_picture_syntax_t& syn = w.syn;
    syn.num_tus = (int32_t)w.tus.size();
    syn.tus = w.tus.data();
    syn.num_coeffs = w.coeffs.size();
    syn.coeffs = w.coeffs.data();
    syn.num_pus = (int32_t)w.pus.size();
    syn.pus = w.pus.data();
    syn.num_wp = (int32_t)w.wp.size();
    syn.wp = w.wp.data();
    syn.blk = w.blk.data();
    syn.sao = w.sao.data();
    syn.ctb_slice = w.ctb_slice.data();
    syn.ctb_tile = w.has_tiles ? w.ctb_tile.data() : nullptr;
    syn.num_slices = (int32_t)w.slices.size();
    syn.slices = w.slices.data();
    syn.scaling = w.has_scaling ? &w.scaling : nullptr;

    if (!deferred) {
        if (run(w)) raise();
        w.clear();
        return;
    }
    // hand the records to the worker and keep parsing; at most two pictures wait
    std::unique_ptr<Work> next;
    {
        const auto t0 = std::chrono::steady_clock::now();
        std::unique_lock<std::mutex> g(q_mu);
        idle_cv.wait(g, [&] { return queue.size() < 2 || !error.empty(); });
        wait_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
        if (!error.empty()) {
            g.unlock();
            raise();
        }
        queue.push_back(std::move(cur));
        if (!spare.empty()) {
            next = std::move(spare.back());
            spare.pop_back();
        }
        if (!worker.joinable()) worker = std::thread([this] { worker_loop(); });
    }
    q_cv.notify_all();
    cur = next ? std::move(next) : std::unique_ptr<Work>(new Work());
}

}  // namespace dropin

// ---- the reference's hooks --------------------------------------------------------------

// The data of a slice segment (coding_tree.cpp:536).  With WPP the reference decodes the
// CTU rows on its thread pool (coding_tree.cpp:404-533), each row starting once the row
// above has finished its second CTU, from the slice's first row to the picture's last, each
// from column 0.  A picture one CTU wide has no second CTU, and every row would wait for
// good; a picture of several slice segments has segments that start inside a row or end
// before the picture does, which that path decodes from the wrong substreams.  Such
// pictures take the reference's sequential path (no thread pool), which follows 9.3.1:
// contexts initialised at a slice and synchronised at a row start within one (initialised
// there when the CTU above and to the right is unavailable, as in a picture one CTU wide).
extern "C" bool __real__ZN4hevc25decode_slice_segment_dataERNS_15DecodingContextERNS_15BitstreamReaderERKSt6vectorImSaImEEm(
    DecodingContext&, hevc::BitstreamReader&, const std::vector<size_t>&, size_t);
extern "C" bool __wrap__ZN4hevc25decode_slice_segment_dataERNS_15DecodingContextERNS_15BitstreamReaderERKSt6vectorImSaImEEm(
    DecodingContext& ctx, hevc::BitstreamReader& bs, const std::vector<size_t>& epb, size_t header_size) {
    hevc::ThreadPool* pool = ctx.thread_pool;
    if (pool && ctx.pps && ctx.pps->entropy_coding_sync_enabled_flag && ctx.sps &&
        (ctx.sps->PicWidthInCtbsY == 1 || ctx.num_slices > 1)) {
        ctx.thread_pool = nullptr;
        bool ok;
        try {
            ok = __real__ZN4hevc25decode_slice_segment_dataERNS_15DecodingContextERNS_15BitstreamReaderERKSt6vectorImSaImEEm(
                ctx, bs, epb, header_size);
        } catch (...) {
            ctx.thread_pool = pool;
            throw;
        }
        ctx.thread_pool = pool;
        return ok;
    }
    return __real__ZN4hevc25decode_slice_segment_dataERNS_15DecodingContextERNS_15BitstreamReaderERKSt6vectorImSaImEEm(
        ctx, bs, epb, header_size);
}

// RefPicList construction (dpb.cpp:245), called for each P and B slice.  A P or B slice
// needs a current reference picture (NumPicTotalCurr > 0, 7.4.7.2); without one the
// reference's list construction loops without end (dpb.cpp:259-266, a damaged stream can
// ask for it), so the drop-in counts NumPicTotalCurr (7-55) from the slice's RPS first and
// refuses the picture instead.
extern "C" void __real__ZN4hevc3DPB23construct_ref_pic_listsERKNS_11SliceHeaderERKNS_3SPSERKNS_3PPSE(
    hevc::DPB*, const hevc::SliceHeader&, const hevc::SPS&, const hevc::PPS&);
extern "C" void __wrap__ZN4hevc3DPB23construct_ref_pic_listsERKNS_11SliceHeaderERKNS_3SPSERKNS_3PPSE(
    hevc::DPB* dpb, const hevc::SliceHeader& sh, const hevc::SPS& sps, const hevc::PPS& pps) {
    if (sh.slice_type != hevc::SliceType::I) {
        const hevc::ShortTermRefPicSet* rps = &sh.st_rps;
        if (sh.short_term_ref_pic_set_sps_flag)
            rps = sh.short_term_ref_pic_set_idx < sps.st_ref_pic_sets.size() ? &sps.st_ref_pic_sets[sh.short_term_ref_pic_set_idx]
                                                                           : nullptr;
        int total = 0;
        if (rps) {
            for (uint32_t i = 0; i < rps->NumNegativePics && i < 16; i++) total += rps->UsedByCurrPicS0[i];
            for (uint32_t i = 0; i < rps->NumPositivePics && i < 16; i++) total += rps->UsedByCurrPicS1[i];
        }
        const uint32_t n_lt = std::min<uint32_t>(32, sh.num_long_term_sps + sh.num_long_term_pics);
        for (uint32_t i = 0; i < n_lt; i++)
            total += i < sh.num_long_term_sps ? sps.used_by_curr_pic_lt_sps_flag[sh.lt_idx_sps[i] % 32]
                                              : sh.used_by_curr_pic_lt_flag[i];
        if (total == 0) {
            dropin::Backend* b = dropin::lookup(dpb);
            b->fail("a P or B slice without a current reference picture (NumPicTotalCurr 0: a damaged stream)");
            b->raise();
        }
    }
    __real__ZN4hevc3DPB23construct_ref_pic_listsERKNS_11SliceHeaderERKNS_3SPSERKNS_3PPSE(dpb, sh, sps, pps);
}

namespace hevc {
void decode_residual_coding(DecodingContext& ctx, int x0, int y0, int log2TrafoSize, int cIdx, int16_t* coefficients);
}

// The levels of a TU, as residual_coding.cpp:175 produces them (x0, y0 in luma samples).
extern "C" void __real__ZN4hevc22decode_residual_codingERNS_15DecodingContextEiiiiPs(DecodingContext&, int, int, int,
                                                                                      int, int16_t*);
extern "C" void __wrap__ZN4hevc22decode_residual_codingERNS_15DecodingContextEiiiiPs(DecodingContext& ctx, int x0,
                                                                                      int y0, int log2, int cIdx,
                                                                                      int16_t* coefficients) {
    __real__ZN4hevc22decode_residual_codingERNS_15DecodingContextEiiiiPs(ctx, x0, y0, log2, cIdx, coefficients);
    const int sub = cIdx ? 2 : 1, n = 1 << log2;
    dropin::Pending& P = dropin::t_pending;
    P.active = true;
    P.t = hevc_tu_t{};
    P.t.x = (uint16_t)(x0 / sub);
    P.t.y = (uint16_t)(y0 / sub);
    P.t.log2_size = (uint8_t)log2;
    P.t.c_idx = (uint8_t)cIdx;
    P.t.flags = HEVC_TU_CODED;
    P.n = n * n;
    std::memcpy(P.lv, coefficients, sizeof(int16_t) * (size_t)P.n);
    P.b = dropin::lookup(ctx.dpb);
    const hevc::CUInfo& cu = ctx.cu_at(x0, y0);
    if (cu.cu_transquant_bypass) {
        // the coding tree copies these levels as the residual and calls no dequantisation
        // or transform hook; an inter TU is complete here, an intra one completes at its
        // prediction
        P.t.flags |= HEVC_TU_BYPASS;
        if (cu.pred_mode != hevc::PredMode::MODE_INTRA) {
            P.b->append_tu(P.t, P.lv, P.n);
            P.active = false;
        }
    }
}

namespace hevc {

void perform_dequant(DecodingContext& ctx, int x0, int y0, int log2, int cIdx, int qp, const int16_t* coefficients,
                     int16_t* scaled) {
    (void)coefficients;
    (void)scaled;
    dropin::Pending& P = dropin::t_pending;
    const int sub = cIdx ? 2 : 1;
    if (!P.active || P.t.c_idx != cIdx || P.t.x != x0 / sub || P.t.y != y0 / sub || P.t.log2_size != log2)
        dropin::lookup(ctx.dpb)->note_unsupported("dequantisation of levels the residual syntax did not produce");
    P.t.qp = (uint8_t)qp;
}

void perform_transform_inverse(int log2, int cIdx, bool is_intra, bool transform_skip, int bit_depth,
                               const int16_t* scaled, int16_t* residual) {
    (void)log2;
    (void)cIdx;
    (void)bit_depth;
    (void)scaled;
    (void)residual;
    dropin::Pending& P = dropin::t_pending;
    if (!P.active) return;
    if (transform_skip) P.t.flags |= HEVC_TU_TSKIP;
    if (!is_intra) {   // an inter TU is complete: its prediction is the PU's
        P.active = false;
        P.b->append_tu(P.t, P.lv, P.n);   // this hook has no context: the decoder of the levels
    }
}

void perform_intra_prediction(DecodingContext& ctx, int x0, int y0, int log2, int cIdx, int mode, int16_t* pred) {
    (void)pred;   // the coding tree zero-fills it; the GPU predicts
    dropin::Backend* b = dropin::lookup(ctx.dpb);
    dropin::Pending& P = dropin::t_pending;
    const int sub = cIdx ? 2 : 1;
    hevc_tu_t t{};
    if (P.active && P.t.c_idx == cIdx && P.t.x == x0 / sub && P.t.y == y0 / sub && P.t.log2_size == log2) {
        t = P.t;
        P.active = false;
    } else {   // an intra TU without levels
        if (P.active) b->note_unsupported("levels without a matching prediction");
        P.active = false;
        t.x = (uint16_t)(x0 / sub);
        t.y = (uint16_t)(y0 / sub);
        t.log2_size = (uint8_t)log2;
        t.c_idx = (uint8_t)cIdx;
    }
    t.flags |= HEVC_TU_INTRA;
    t.intra_mode = (uint8_t)mode;
    b->append_tu(t, P.lv, (t.flags & HEVC_TU_CODED) ? (1 << (2 * log2)) : 0);
}

void perform_inter_prediction(DecodingContext& ctx, int xPb, int yPb, int w, int h, int cIdx, const MV& mv0,
                              const MV& mv1, int ref0, int ref1, bool pf0, bool pf1, int16_t* pred) {
    // the coding tree copies `pred` into its own picture, which the GPU's samples replace
    // at the end of the picture; give it defined values
    const int sub = cIdx ? 2 : 1;
    std::memset(pred, 0, sizeof(int16_t) * (size_t)(w / sub) * (size_t)(h / sub));
    if (cIdx != 0) return;
    dropin::Backend* b = dropin::lookup(ctx.dpb);
    hevc_pu_t u{};
    u.x = (uint16_t)xPb;
    u.y = (uint16_t)yPb;
    u.w = (uint8_t)w;
    u.h = (uint8_t)h;
    u.ref_idx[0] = (int8_t)(pf0 ? ref0 : -1);
    u.ref_idx[1] = (int8_t)(pf1 ? ref1 : -1);
    u.mv[0][0] = (int16_t)mv0.x;
    u.mv[0][1] = (int16_t)mv0.y;
    u.mv[1][0] = (int16_t)mv1.x;
    u.mv[1][1] = (int16_t)mv1.y;
    u.wp = -1;
    // explicit weighted prediction of the PU's slice (interpolation.cpp:392-400, :246-300)
    const SliceHeader& sh = *ctx.sh;
    const bool wpf = (sh.slice_type == SliceType::P && ctx.pps->weighted_pred_flag) ||
                     (sh.slice_type == SliceType::B && ctx.pps->weighted_bipred_flag);
    hevc_wp_t wt{};
    if (wpf) {
        const PredWeightTable& t = sh.pred_weight_table;
        wt.log2wd[0] = (int16_t)(t.luma_log2_weight_denom + 6);
        wt.log2wd[1] = (int16_t)((int)t.luma_log2_weight_denom + t.delta_chroma_log2_weight_denom + 6);
        const PredWeightTable::RefWeight* rw[2] = {&t.l0[(size_t)(ref0 >= 0 ? ref0 : 0)],
                                                   &t.l1[(size_t)(ref1 >= 0 ? ref1 : 0)]};
        for (int l = 0; l < 2; l++) {
            wt.w[l][0] = rw[l]->luma_weight;
            wt.o[l][0] = rw[l]->luma_offset;
            for (int c = 0; c < 2; c++) {
                wt.w[l][c + 1] = rw[l]->chroma_weight[c];
                wt.o[l][c + 1] = rw[l]->chroma_offset[c];
            }
        }
    }
    const Picture* rp[2] = {pf0 ? ctx.dpb->ref_pic_list0(ref0) : nullptr, pf1 ? ctx.dpb->ref_pic_list1(ref1) : nullptr};
    std::lock_guard<std::mutex> g(b->rec_mu);
    dropin::Work& wk = *b->cur;
    if (wpf) {
        u.wp = (int16_t)wk.wp.size();
        wk.wp.push_back(wt);
    }
    wk.pus.push_back(u);
    wk.pu_ref[0].push_back(rp[0]);
    wk.pu_ref[1].push_back(rp[1]);
}

void apply_deblocking(DecodingContext& ctx) { dropin::lookup(ctx.dpb)->finish_records(ctx); }

void apply_sao(DecodingContext& ctx) { dropin::lookup(ctx.dpb)->submit(ctx); }

}  // namespace hevc
