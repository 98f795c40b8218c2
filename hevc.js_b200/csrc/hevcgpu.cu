// hevcgpu.cu — host side of the B200 reconstruction back end: context, pooled device
// memory, DPB slots in HBM, picture jobs (validation, binning, per-CTU intra lists,
// wavefront diagonals), launch sequencing, and the C ABI of include/hevcgpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "hevcgpu.h"
#include "intra.cuh"
#include "mc.cuh"
#include "kernels.cuh"

using namespace hevcgpu;

// ---------------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------------
namespace {
thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(HEVCGPU_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

struct Layout {  // pitched 8-bit 4:2:0 picture buffer
    int32_t W = 0, H = 0, pitch_y = 0, pitch_c = 0;
    int64_t off_cb = 0, off_cr = 0, bytes = 0;
    void init(int w, int h) {
        W = w;
        H = h;
        pitch_y = (int32_t)align_up(w, 64);
        pitch_c = (int32_t)align_up(w / 2, 64);
        off_cb = (int64_t)pitch_y * h;
        off_cr = off_cb + (int64_t)pitch_c * (h / 2);
        bytes = align_up(off_cr + (int64_t)pitch_c * (h / 2), 256);
    }
};

// Persistent host workers.  run(n, f) calls f(i) for every i < n, spread over the
// workers and the calling thread, and returns when all calls are done.  One run at a
// time per pool (the caller holds run_mu).  Workers make the context's device current
// once at start.
class HostPool {
  public:
    ~HostPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    // Starts the workers on first use; false if no thread could be started.
    void ensure(int device) {
        std::lock_guard<std::mutex> g(m_);
        if (started_) return;
        started_ = true;
        unsigned hw = std::thread::hardware_concurrency();
        int workers = (int)std::min<unsigned>(hw ? hw : 1, 64) - 1;
        for (int i = 0; i < workers; i++) {
            try {
                threads_.emplace_back([this, device] { loop(device); });
            } catch (...) {
                break;
            }
        }
    }
    void run(int n, const std::function<void(int)>& f) {
        if (n <= 0) return;
        std::unique_lock<std::mutex> lk(m_);
        task_ = &f;
        n_ = n;
        next_.store(0);
        done_ = 0;
        gen_++;
        lk.unlock();
        cv_.notify_all();
        int finished = drain(f);
        lk.lock();
        done_ += finished;
        done_cv_.wait(lk, [&] { return done_ == n_ && busy_ == 0; });
        task_ = nullptr;
    }
    std::mutex run_mu;

  private:
    int drain(const std::function<void(int)>& f) {
        int finished = 0;
        for (int i = next_.fetch_add(1); i < n_; i = next_.fetch_add(1)) {
            f(i);
            finished++;
        }
        return finished;
    }
    void loop(int device) {
        cudaSetDevice(device);
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            cv_.wait(lk, [&] { return stop_ || (gen_ != seen && task_); });
            if (stop_) return;
            seen = gen_;
            const std::function<void(int)>* f = task_;
            busy_++;
            lk.unlock();
            int finished = drain(*f);
            lk.lock();
            busy_--;
            done_ += finished;
            if (done_ == n_ && busy_ == 0) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* task_ = nullptr;
    std::atomic<int> next_{0};
    int n_ = 0, done_ = 0, busy_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false, started_ = false;
};

}  // namespace

// ---------------------------------------------------------------------------------------
// context and device memory pool
// ---------------------------------------------------------------------------------------
struct hevcgpu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t budget = ~0ull;
    uint64_t allocated = 0;       // bytes obtained from cudaMalloc (pooled or in use)
    uint64_t launches = 0;
    std::multimap<size_t, void*> free_blocks;
    std::map<void*, size_t> sizes;
    std::mutex mu;
    // stage profiling
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    struct Mark { int stage; cudaEvent_t a, b; uint64_t launches; };
    std::vector<Mark> marks;

    cudaEvent_t next_event() {
        if (ev_used == ev_pool.size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }

    int alloc(void** p, size_t bytes) {
        bytes = (size_t)align_up((int64_t)std::max<size_t>(bytes, 256), 4096);
        std::lock_guard<std::mutex> g(mu);
        auto it = free_blocks.lower_bound(bytes);
        if (it != free_blocks.end() && it->first <= bytes * 2) {
            *p = it->second;
            free_blocks.erase(it);
            return HEVCGPU_OK;
        }
        if (allocated + bytes > budget) {
            // give pooled blocks back before refusing
            for (auto& fb : free_blocks) {
                cudaFree(fb.second);
                allocated -= fb.first;
                sizes.erase(fb.second);
            }
            free_blocks.clear();
            if (allocated + bytes > budget)
                return fail(HEVCGPU_ENOMEM, "HBM budget exceeded: %llu in use + %llu > %llu",
                            (unsigned long long)allocated, (unsigned long long)bytes, (unsigned long long)budget);
        }
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(HEVCGPU_ENOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
        }
        allocated += bytes;
        sizes[*p] = bytes;
        return HEVCGPU_OK;
    }
    void release(void* p) {
        if (!p) return;
        std::lock_guard<std::mutex> g(mu);
        auto it = sizes.find(p);
        if (it == sizes.end()) return;
        free_blocks.emplace(it->second, p);
    }
    // pinned host staging pool (record images and picture descriptors)
    std::multimap<size_t, void*> free_host;
    std::map<void*, size_t> host_sizes;
    int alloc_host(void** p, size_t bytes) {
        bytes = (size_t)align_up((int64_t)std::max<size_t>(bytes, 4096), 65536);
        std::lock_guard<std::mutex> g(mu);
        auto it = free_host.lower_bound(bytes);
        if (it != free_host.end() && it->first <= bytes * 2) {
            *p = it->second;
            free_host.erase(it);
            return HEVCGPU_OK;
        }
        cudaError_t e = cudaHostAlloc(p, bytes, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(HEVCGPU_ENOMEM, "cudaHostAlloc(%zu): %s", bytes, cudaGetErrorString(e));
        }
        host_sizes[*p] = bytes;
        return HEVCGPU_OK;
    }
    void release_host(void* p) {
        if (!p) return;
        std::lock_guard<std::mutex> g(mu);
        auto it = host_sizes.find(p);
        if (it != host_sizes.end()) free_host.emplace(it->second, p);
    }
    // host worker pool for the batched host-side calls (job preparation, downloads)
    HostPool pool;
    std::vector<cudaEvent_t> dl_events;  // per-picture completion of batched downloads
    // intra CTU tasks: FlowState, the sticky status word (16 bytes on), and one ticket
    // counter per picture of a launch (32 bytes on)
    void* flow = nullptr;
    static constexpr size_t FLOW_BYTES = sizeof(FlowState) + 16 + sizeof(int32_t) * MAX_SEGS;
    int32_t* tickets() { return reinterpret_cast<int32_t*>(static_cast<uint8_t*>(flow) + sizeof(FlowState) + 16); }
    int sm_count = 148;
    // completion events of the batches on the context's own stream, used in turn: a job
    // waits for its own batch's event (re-recorded only EVENT_RING batches later)
    static constexpr int EVENT_RING = 16;
    cudaEvent_t done[EVENT_RING] = {};
    int done_next = 0;
    cudaEvent_t next_done() { cudaEvent_t e = done[done_next]; done_next = (done_next + 1) % EVENT_RING; return e; }
    std::mutex jobs_mu;
    std::set<hevcgpu_job*> live_jobs;   // jobs of the DPB API, for lanes that close
    // Reads and clears the sticky device status of a flow area; maps it to a return code.
    int take_status() { return take_status_of(flow); }
    static int take_status_of(void* flow_area) {
        uint32_t st = 0;
        uint32_t* sticky = reinterpret_cast<uint32_t*>(static_cast<FlowState*>(flow_area) + 1);
        if (cudaMemcpy(&st, sticky, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(HEVCGPU_ECUDA, "reading the device status: %s", cudaGetErrorString(cudaGetLastError()));
        if (!st) return HEVCGPU_OK;
        cudaMemset(sticky, 0, sizeof(uint32_t));
        if (st & ST_TIMEOUT) return fail(HEVCGPU_ETIMEOUT, "a bounded device wait gave up (status 0x%x)", st);
        return fail(HEVCGPU_EDEVICE, "a kernel refused a record (status 0x%x)", st);
    }
    ~hevcgpu_ctx() {
        if (flow) cudaFree(flow);
        for (auto e : done)
            if (e) cudaEventDestroy(e);
        for (auto e : ev_pool) cudaEventDestroy(e);
        for (auto e : dl_events) cudaEventDestroy(e);
        for (auto& h : host_sizes) cudaFreeHost(h.first);
        for (auto& s : sizes) cudaFree(s.first);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

struct DevBuf {  // pooled device buffer
    hevcgpu_ctx* ctx = nullptr;
    void* p = nullptr;
    size_t n = 0;
    int get(hevcgpu_ctx* c, size_t bytes) {
        if (p && n >= bytes) return HEVCGPU_OK;
        put();
        ctx = c;
        int rc = c->alloc(&p, bytes);
        if (rc == HEVCGPU_OK) n = bytes;
        return rc;
    }
    void put() {
        if (p && ctx) ctx->release(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { put(); }
};

struct HostBuf {  // pooled pinned host buffer
    hevcgpu_ctx* ctx = nullptr;
    void* p = nullptr;
    size_t n = 0;
    int get(hevcgpu_ctx* c, size_t bytes) {
        if (p && n >= bytes) return HEVCGPU_OK;
        put();
        ctx = c;
        int rc = c->alloc_host(&p, bytes);
        if (rc == HEVCGPU_OK) n = bytes;
        return rc;
    }
    void put() {
        if (p && ctx) ctx->release_host(p);
        p = nullptr;
        n = 0;
    }
    ~HostBuf() { put(); }
};

}  // namespace

struct hevcgpu_lane {
    hevcgpu_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    void* flow = nullptr;              // FlowState, status word, per-picture tickets
    cudaEvent_t done[hevcgpu_ctx::EVENT_RING] = {};   // batch completion events, used in turn
    int done_next = 0;
    cudaEvent_t ctx_ready = nullptr;   // the context stream's work before a batch
    // Asynchronous downloads run on a stream of their own after the lane's work queued
    // before them (src_ready), so the lane's next batches do not queue behind the copies.
    cudaStream_t cstream = nullptr;
    cudaEvent_t src_ready = nullptr;
    // Asynchronous downloads: download k (k = 1, 2, ...) records dl_done[k % EVENT_RING]
    // after its copies; a later download reuses the slot, whose event then completes later,
    // so waiting on it still waits for download k.
    cudaEvent_t dl_done[hevcgpu_ctx::EVENT_RING] = {};
    uint64_t dl_seq = 0;
    cudaEvent_t next_done() {
        cudaEvent_t e = done[done_next];
        done_next = (done_next + 1) % hevcgpu_ctx::EVENT_RING;
        return e;
    }
    ~hevcgpu_lane() {
        if (stream) cudaStreamSynchronize(stream);
        if (flow) cudaFree(flow);
        for (auto e : done)
            if (e) cudaEventDestroy(e);
        if (cstream) cudaStreamSynchronize(cstream);
        for (auto e : dl_done)
            if (e) cudaEventDestroy(e);
        if (ctx_ready) cudaEventDestroy(ctx_ready);
        if (src_ready) cudaEventDestroy(src_ready);
        if (cstream) cudaStreamDestroy(cstream);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct hevcgpu_stream {
    hevcgpu_ctx* ctx = nullptr;
    Layout lay;
    std::vector<DevBuf> slots;
    // Per slot: an event recorded on a lane's copy stream after the last asynchronous
    // download of the slot (or null); a launch or upload that writes the slot first waits
    // for it on the device.
    std::vector<cudaEvent_t> slot_read;
    ~hevcgpu_stream() {
        for (cudaEvent_t e : slot_read)
            if (e) {
                cudaEventSynchronize(e);   // no copy may still read a slot being released
                cudaEventDestroy(e);
            }
    }
    // Orders `stream` after the downloads still reading slot k.
    int wait_slot_read(int k, cudaStream_t stream) {
        if (k < 0 || k >= (int)slot_read.size() || !slot_read[(size_t)k]) return HEVCGPU_OK;
        return cudaStreamWaitEvent(stream, slot_read[(size_t)k], 0) == cudaSuccess ? HEVCGPU_OK : HEVCGPU_ECUDA;
    }
};

// ---------------------------------------------------------------------------------------
// jobs: one picture's records, prepared and uploaded
// ---------------------------------------------------------------------------------------
// A CUDA call of a job's preparation: a host->device copy, zeroing device memory, or
// recording the event that marks the copies straight from the caller's arrays as done.
// Prepared on the context's host workers, the calls are queued in the job and issued by
// the thread that asked for the batch, so that the workers make no CUDA calls (which would
// contend for the driver's locks) and every upload goes out from one thread in order.
struct UploadOp {
    enum Kind : int { COPY, ZERO, MARK_DIRECT } kind;
    void* dst;
    const void* src;
    size_t bytes;
};

struct hevcgpu_job {
    hevcgpu_ctx* ctx = nullptr;
    hevcgpu_stream* st = nullptr;  // may be null for stage entry points
    Layout lay;
    DevBuf recs;      // the small record arrays + work lists, one upload
    DevBuf big;       // the caller's large arrays: PUs, 4x4 grid, TUs, coefficient levels
    HostBuf pin_big;  // pinned staging for those of them not in page-locked memory
    DevBuf rec;       // reconstruction / deblocking buffer (pitched picture)
    DevBuf scratch;   // resid (int16) + motion grid
    DevBuf desc;      // PicDesc
    HostBuf pin;      // pinned staging: the record image, then the PicDesc
    size_t desc_off = 0;
    cudaEvent_t desc_copied = nullptr;  // the last PicDesc upload has read the staging copy
    cudaEvent_t direct_read = nullptr;  // the uploads straight from the caller's arrays are done
    PicDesc host_desc{};
    int32_t n_res[4] = {0, 0, 0, 0};
    const int32_t* d_res[4] = {nullptr, nullptr, nullptr, nullptr};
    int32_t n_mc[2] = {0, 0};            // luma strips, chroma strips (mc.cuh items)
    const uint32_t* d_mc[2] = {nullptr, nullptr};
    int32_t n_ictu = 0;                 // CTUs that hold intra TUs
    uint32_t spare_dep = 0;             // dependency list entry kept for the planted wait
    int32_t epoch = 0;                  // intra launches of this job so far
    int32_t n_pus = 0;
    int has_intra = 0;
    int32_t dst_slot = -2;              // slot currently written into host_desc / desc
    cudaStream_t last_stream = nullptr; // stream of the job's last launch (null: the context's)
    cudaEvent_t last_done = nullptr;    // recorded after that launch
    bool registered = false;            // in ctx->live_jobs
    uint64_t upload_bytes = 0;          // host -> device bytes of the prepare call
    std::vector<UploadOp> ops;          // CUDA calls of the preparation not yet issued
    hevc_pic_params_t params{};
    ~hevcgpu_job() {
        // buffers go back to the pools only after every queued use of them has run: a job's
        // uploads all precede its launches (the launching stream waits for the context
        // stream, and descriptor copies go on the launching stream), so the completion of its
        // last batch covers them; a job never launched waits for the context stream
        if (last_done) cudaEventSynchronize(last_done);   // the job's last batch, not later ones
        else if (last_stream) cudaStreamSynchronize(last_stream);
        else if (ctx) cudaStreamSynchronize(ctx->stream);
        if (registered) {
            std::lock_guard<std::mutex> g(ctx->jobs_mu);
            ctx->live_jobs.erase(this);
        }
        if (desc_copied) cudaEventDestroy(desc_copied);
        if (direct_read) cudaEventDestroy(direct_read);
    }
};

namespace {

// Host image of a job's device records: offsets into one buffer.  A first pass with
// out == nullptr only measures; the second pass writes into pinned staging memory.
struct Packer {
    uint8_t* out = nullptr;
    size_t size = 0;
    size_t add(const void* src, size_t bytes) {
        size_t off = (size_t)align_up((int64_t)size, 256);
        size = off + bytes;
        if (out && bytes && src) std::memcpy(out + off, src, bytes);
        return off;
    }
};

// True when p points into page-locked host memory (cudaHostAlloc or registered).
bool page_locked(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    const bool ok = cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return ok;
}

// Branch-free screens of the TU and PU arrays: true when every record passes the checks
// of validate(); validate() walks the records one by one (to name the first bad one) only
// when a screen fails.
bool tus_pass(const hevc_picture_syntax_t* s, int W, int H) {
    uint32_t bad = 0;
    const uint32_t ncoef = (uint32_t)s->num_coeffs;
    for (int i = 0; i < s->num_tus; i++) {
        const hevc_tu_t& t = s->tus[i];
        const uint32_t lg = t.log2_size & 7u, n = 1u << lg;
        const uint32_t pw = t.c_idx ? (uint32_t)W / 2 : (uint32_t)W, ph = t.c_idx ? (uint32_t)H / 2 : (uint32_t)H;
        bad |= (uint32_t)(t.log2_size - 2u > 3u) | (uint32_t)(t.c_idx > 2) | (uint32_t)(((t.x | t.y) & (n - 1)) != 0) |
               (uint32_t)(t.x + n > pw) | (uint32_t)(t.y + n > ph) |
               (uint32_t)((t.flags & HEVC_TU_INTRA) && t.intra_mode > 34) |
               (uint32_t)((t.flags & HEVC_TU_PCM) && (~t.flags & (HEVC_TU_INTRA | HEVC_TU_CODED)));
        const uint64_t end = (uint64_t)t.coeff_offset + (uint64_t)n * n;
        bad |= (uint32_t)((t.flags & HEVC_TU_CODED) && ((t.coeff_offset & 15) | (uint32_t)(end > ncoef) |
                                                        (uint32_t)(t.qp > 51 + 48)));
    }
    return bad == 0;
}
bool pus_pass(const hevc_picture_syntax_t* s, int W, int H) {
    uint32_t bad = 0;
    const int n0 = s->params.num_ref[0], n1 = s->params.num_ref[1];
    for (int i = 0; i < s->num_pus; i++) {
        const hevc_pu_t& u = s->pus[i];
        bad |= (uint32_t)(u.w - 4u > 60u) | (uint32_t)(u.h - 4u > 60u) | ((u.w | u.h | u.x | u.y) & 3u) |
               (uint32_t)(u.x + u.w > W) | (uint32_t)(u.y + u.h > H) |
               (uint32_t)(u.ref_idx[0] < 0 && u.ref_idx[1] < 0) | (uint32_t)(u.ref_idx[0] >= n0) |
               (uint32_t)(u.ref_idx[1] >= n1) | (uint32_t)(u.wp >= s->num_wp);
    }
    return bad == 0;
}

int validate(const hevc_picture_syntax_t* s, bool need_tus, bool need_pus, bool need_filters) {
    if (!s) return fail(HEVCGPU_EINVAL, "null picture syntax");
    const hevc_pic_params_t& p = s->params;
    if (p.bit_depth != 8) return fail(HEVCGPU_EUNSUPPORTED, "bit depth %d (only 8 is supported)", p.bit_depth);
    if (p.width <= 0 || p.height <= 0 || (p.width & 7) || (p.height & 7) || p.width > 8192 || p.height > 8192)
        return fail(HEVCGPU_EINVAL, "picture size %dx%d (multiples of 8 up to 8192)", p.width, p.height);
    if (p.log2_ctb < 4 || p.log2_ctb > 6) return fail(HEVCGPU_EUNSUPPORTED, "log2_ctb %d", p.log2_ctb);
    if (p.log2_min_tb != 2) return fail(HEVCGPU_EUNSUPPORTED, "log2_min_tb %d (4x4 minimum TB)", p.log2_min_tb);
    for (int l = 0; l < 2; l++)
        if (p.num_ref[l] < 0 || p.num_ref[l] > 16) return fail(HEVCGPU_EINVAL, "num_ref[%d] = %d", l, p.num_ref[l]);
    const int W = p.width, H = p.height;
    if (need_tus) {
        if (s->num_tus < 0 || (s->num_tus && !s->tus)) return fail(HEVCGPU_EINVAL, "bad TU array");
        for (int i = tus_pass(s, W, H) ? s->num_tus : 0; i < s->num_tus; i++) {
            const hevc_tu_t& t = s->tus[i];
            int n = 1 << t.log2_size, sub = t.c_idx ? 2 : 1;
            if (t.log2_size < 2 || t.log2_size > 5 || t.c_idx > 2 || (t.x % n) || (t.y % n) ||
                t.x + n > W / sub || t.y + n > H / sub)
                return fail(HEVCGPU_EINVAL, "TU %d at (%d,%d) size %d comp %d is outside the picture or unaligned", i,
                            t.x, t.y, n, t.c_idx);
            if ((t.flags & HEVC_TU_INTRA) && t.intra_mode > 34)
                return fail(HEVCGPU_EINVAL, "TU %d intra mode %d", i, t.intra_mode);
            if ((t.flags & HEVC_TU_PCM) && (~t.flags & (HEVC_TU_INTRA | HEVC_TU_CODED)))
                return fail(HEVCGPU_EINVAL, "TU %d is PCM but not an intra TU with levels", i);
            if (t.flags & HEVC_TU_CODED) {
                if ((t.coeff_offset & 15) || (uint64_t)t.coeff_offset + (uint64_t)n * n > s->num_coeffs)
                    return fail(HEVCGPU_EINVAL, "TU %d coeff_offset %u (multiple of 16, inside the pool)", i,
                                t.coeff_offset);
                if (t.qp > 51 + 48) return fail(HEVCGPU_EINVAL, "TU %d qp %d", i, t.qp);
            }
        }
    }
    if (need_pus) {
        if (s->num_pus < 0 || (s->num_pus && !s->pus)) return fail(HEVCGPU_EINVAL, "bad PU array");
        if (s->num_pus > MC_MAX_PUS) return fail(HEVCGPU_EINVAL, "%d PUs, at most %d", s->num_pus, MC_MAX_PUS);
        for (int i = pus_pass(s, W, H) ? s->num_pus : 0; i < s->num_pus; i++) {
            const hevc_pu_t& u = s->pus[i];
            if (u.w < 4 || u.h < 4 || u.w > 64 || u.h > 64 || (u.w & 3) || (u.h & 3) || (u.x & 3) || (u.y & 3) ||
                u.x + u.w > W || u.y + u.h > H)
                return fail(HEVCGPU_EINVAL, "PU %d (%d,%d %dx%d) outside the picture", i, u.x, u.y, u.w, u.h);
            if (u.ref_idx[0] < 0 && u.ref_idx[1] < 0) return fail(HEVCGPU_EINVAL, "PU %d uses no list", i);
            for (int l = 0; l < 2; l++)
                if (u.ref_idx[l] >= p.num_ref[l]) return fail(HEVCGPU_EINVAL, "PU %d refIdxL%d %d", i, l, u.ref_idx[l]);
            if (u.wp >= s->num_wp) return fail(HEVCGPU_EINVAL, "PU %d WP row %d", i, u.wp);
        }
        for (int i = 0; i < s->num_wp; i++)
            for (int c = 0; c < 2; c++)
                if (s->wp[i].log2wd[c] < 1 || s->wp[i].log2wd[c] > 20)
                    return fail(HEVCGPU_EINVAL, "WP row %d log2wd %d", i, s->wp[i].log2wd[c]);
    }
    if (need_filters) {
        if (!s->blk) return fail(HEVCGPU_EINVAL, "missing 4x4 side-information grid");
        if (!s->sao && p.sao_enabled) return fail(HEVCGPU_EINVAL, "missing SAO parameters");
        if (s->num_slices < 1 || !s->slices) return fail(HEVCGPU_EINVAL, "missing slice parameters");
        int ctb = 1 << p.log2_ctb;
        int nctb = ((W + ctb - 1) / ctb) * ((H + ctb - 1) / ctb);
        if (s->ctb_slice)
            for (int a = 0; a < nctb; a++)
                if (s->ctb_slice[a] >= s->num_slices) return fail(HEVCGPU_EINVAL, "CTB %d slice index", a);
        if (s->sao)
            for (int a = 0; a < nctb; a++)
                for (int c = 0; c < 3; c++)
                    if (s->sao[a].type[c] > 2 || s->sao[a].eo_class[c] > 3 || s->sao[a].band_pos[c] > 31)
                        return fail(HEVCGPU_EINVAL, "CTB %d SAO parameters", a);
    }
    return HEVCGPU_OK;
}

enum StageMask : int {
    ST_MC = 1,
    ST_RESID = 2,
    ST_INTRA = 4,
    ST_DEBLOCK = 8,
    ST_SAO = 16,
    ST_ALL = 31,
};

// Build the host image, upload it and fill host_desc (except dst/ref pointers).
// Work vectors of job_build, kept per host thread (the context's workers live as long as
// the context), so that their memory is reused from one picture to the next: no allocation
// and no first-touch page faults per picture.
struct BuildScratch {
    std::vector<int32_t> bins[4], intra_list, itu, level, ctu_of, order;
    // intra owner maps, one word per 4x4 unit: (generation << 24) | decode-order index of the
    // intra TU.  An entry is valid when its generation is this picture's, so the maps need
    // clearing only when the 8-bit generation wraps.
    std::vector<uint32_t> owner[3];
    uint32_t gen = 0;
    std::vector<hevc_tu_t> itu_rec;
    std::vector<int4> itu_res;
    // intra schedule
    std::vector<int32_t> dep_at, deps, pos, cnt;
    std::vector<std::pair<int64_t, int32_t>> runs;   // (wavefront key, first TU) of each CTU's run
    std::vector<int32_t> ictu_addr, ictu_tu_off, slot_of;
    std::vector<uint32_t> itu_dep, dep_out, watch, ictu_watch;
    std::vector<uint8_t> task_flags;   // hevcgpu_intra_schedule's copy of the tasks' flags
    std::vector<uint32_t> mc[2];
    std::vector<uint8_t> mc_cls;
};
thread_local BuildScratch t_build;

// MC strips: 4 columns x up to 16 rows of one PU in one plane, one thread each; luma
// and chroma (Cb and Cr strips) are two lists, each ordered by class: bi-predicted
// first, then windows inside the picture first, then taller first, so that the
// threads of a warp share their path and row count; PU order inside a class.  One pass
// finds each PU's class word in both planes and counts its strips per class by row
// band; a second pass writes the items of each row band.
void build_mc_strips(BuildScratch& BS, const hevc_picture_syntax_t* s, int pitch_y, int pitch_c) {
    const int W = s->params.width, H = s->params.height;
    auto& mc = BS.mc;
    mc[0].clear();
    mc[1].clear();
    const int n_pu = s->num_pus;
    int32_t cnt[2][33] = {};
    auto& cls = BS.mc_cls;   // per PU and plane: (bi ? 0 : 2) + (inside ? 0 : 1)
    cls.resize((size_t)n_pu * 2);
    for (int i = 0; i < n_pu; i++) {
        const hevc_pu_t& u = s->pus[i];
        const bool bi = u.ref_idx[0] >= 0 && u.ref_idx[1] >= 0;
        const int wl = u.w, hl = u.h, wc = u.w / 2, hc = u.h / 2;
        // list windows at the PU's top-left, extended over the PU: its strips are
        // inside when every list's window of the whole PU is
        bool in_l = true, in_c = true;
        for (int l = 0; l < 2; l++) {
            if (u.ref_idx[l] < 0) continue;
            const int mvx = u.mv[l][0], mvy = u.mv[l][1];
            const int x0 = u.x + (mvx >> 2) - 3, y0 = u.y + (mvy >> 2) - 3;
            in_l = in_l && mc_inside<false>(x0, y0, hl, W, H, pitch_y) &&
                   mc_inside<false>(x0 + ((wl - 1) & ~3), y0, hl, W, H, pitch_y);
            const int cx0 = u.x / 2 + (mvx >> 3) - 1, cy0 = u.y / 2 + (mvy >> 3) - 1;
            in_c = in_c && mc_inside<true>(cx0, cy0, hc, W / 2, H / 2, pitch_c) &&
                   mc_inside<true>(cx0 + ((wc - 1) & ~3), cy0, hc, W / 2, H / 2, pitch_c);
        }
        const int kl = (bi ? 0 : 2) + (in_l ? 0 : 1), kc = (bi ? 0 : 2) + (in_c ? 0 : 1);
        cls[2 * (size_t)i] = (uint8_t)kl;
        cls[2 * (size_t)i + 1] = (uint8_t)kc;
        // class = kind * (row classes) + (row classes) - rows / (rows per class)
        const int nl = wl / 4, nc = 2 * ((wc + 3) / 4);
        for (int sy = 0; sy < hl; sy += MC_STRIP_ROWS)
            cnt[0][kl * 4 + 4 - std::min(MC_STRIP_ROWS, hl - sy) / 4 + 1] += nl;
        for (int sy = 0; sy < hc; sy += MC_STRIP_ROWS)
            cnt[1][kc * 8 + 8 - std::min(MC_STRIP_ROWS, hc - sy) / 2 + 1] += nc;
    }
    for (int c = 0; c < 2; c++) {
        const int ncls = c ? 32 : 16;
        for (int k = 1; k <= ncls; k++) cnt[c][k] += cnt[c][k - 1];
        mc[c].resize((size_t)cnt[c][ncls]);
    }
    uint32_t* out_l = mc[0].data();
    uint32_t* out_c = mc[1].data();
    for (int i = 0; i < n_pu; i++) {
        const hevc_pu_t& u = s->pus[i];
        const int kl = cls[2 * (size_t)i], kc = cls[2 * (size_t)i + 1];
        for (int sy = 0; sy < u.h; sy += MC_STRIP_ROWS) {
            const int rows = std::min(MC_STRIP_ROWS, u.h - sy);
            int32_t& pos = cnt[0][kl * 4 + 4 - rows / 4];
            uint32_t item = mc_item(i, 0, sy, rows, false, 0);
            for (int sx = 0; sx < u.w; sx += 4, item += 1u << 20) out_l[pos++] = item;
        }
        const int wc = u.w / 2, hc = u.h / 2;
        for (int sy = 0; sy < hc; sy += MC_STRIP_ROWS) {
            const int rows = std::min(MC_STRIP_ROWS, hc - sy);
            int32_t& pos = cnt[1][kc * 8 + 8 - rows / 2];
            for (int pl = 0; pl < 2; pl++) {
                uint32_t item = mc_item(i, 0, sy, rows, true, pl);
                for (int sx = 0; sx < wc; sx += 4, item += 1u << 20) out_c[pos++] = item;
            }
        }
    }
}

// Issue one queued CUDA call of a job's preparation on the context stream.
int run_upload(hevcgpu_job* j, const UploadOp& o) {
    cudaStream_t cs = j->ctx->stream;
    switch (o.kind) {
    case UploadOp::COPY:
        CUDA_TRY(cudaMemcpyAsync(o.dst, o.src, o.bytes, cudaMemcpyHostToDevice, cs));
        break;
    case UploadOp::ZERO:
        CUDA_TRY(cudaMemsetAsync(o.dst, 0, o.bytes, cs));
        break;
    case UploadOp::MARK_DIRECT:
        if (!j->direct_read) CUDA_TRY(cudaEventCreateWithFlags(&j->direct_read, cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(j->direct_read, cs));
        break;
    }
    return HEVCGPU_OK;
}

// Issue the calls a deferred job_build queued, in order.
int job_issue(hevcgpu_job* j) {
    int rc = HEVCGPU_OK;
    for (const UploadOp& o : j->ops)
        if ((rc = run_upload(j, o))) break;
    j->ops.clear();
    return rc;
}

// defer: queue the CUDA calls in j->ops (job_issue issues them) instead of making them.
// The intra schedule of a picture (the intra TUs of BS.intra_list, in decode order): the
// CTUs that hold intra TUs in wavefront order, their TUs in task order, each TU's
// dependency list and each CTU's watch list (intra.cuh, k_intra_ctus).  *spare_dep
// receives the index of the spare dependency entry (hevcgpu_job_plant_unmet_wait).
int build_intra_schedule(BuildScratch& BS, const hevc_picture_syntax_t* s, uint32_t* spare_dep) {
    const hevc_pic_params_t& p = s->params;
    const int W = p.width, H = p.height;
    const int ctb = 1 << p.log2_ctb;
    const int wctb = (W + ctb - 1) / ctb, hctb = (H + ctb - 1) / ctb, nctb = wctb * hctb;
    (void)hctb;
    const auto& intra_list = BS.intra_list;
    const int n_intra = (int)intra_list.size();
    auto& ictu_addr = BS.ictu_addr;
    auto& ictu_tu_off = BS.ictu_tu_off;
    auto& itu = BS.itu;
    auto& itu_rec = BS.itu_rec;
    auto& itu_res = BS.itu_res;
    auto& itu_dep = BS.itu_dep;
    auto& dep_out = BS.dep_out;
    auto& ictu_watch = BS.ictu_watch;
    ictu_addr.clear();
    ictu_watch.clear();
    BS.watch.clear();
    ictu_tu_off.clear();
    itu.clear();
    itu_rec.clear();
    itu_res.clear();
    itu_dep.clear();
    dep_out.clear();
    if (!n_intra) return HEVCGPU_OK;
    auto& level = BS.level;
    auto& ctu_of = BS.ctu_of;
    auto& dep_at = BS.dep_at;       // decode order: first entry of TU b's owners in deps
    auto& deps = BS.deps;           // decode-order indices of the owners, per TU
    level.resize((size_t)n_intra);
    ctu_of.resize((size_t)n_intra);
    dep_at.resize((size_t)n_intra + 1);
    // owners found, written through a raw pointer into a buffer kept 34 entries (the most
    // one TU can add) ahead of the count
    size_t n_own = 0;
    if (deps.size() < (size_t)n_intra * 3 + 64) deps.resize((size_t)n_intra * 3 + 64);
    int32_t* D = deps.data();
    // owner maps: the decode-order index of the latest intra TU per 4x4 unit (24 bits),
    // in words tagged with this picture's generation (8 bits; a word of another
    // generation: no owner)
    if (n_intra >= (1 << 24)) return fail(HEVCGPU_EINVAL, "%d intra TUs in one picture", n_intra);
    auto& owner = BS.owner;
    int uw[3], uh[3];
    if (++BS.gen == 256u) {   // wrapped: no old word may carry the new generation
        for (auto& m : owner) std::fill(m.begin(), m.end(), 0u);
        BS.gen = 1;
    }
    const uint32_t gtag = BS.gen << 24;
    constexpr uint32_t GEN_BITS = 0xFF000000u;
    for (int c = 0; c < 3; c++) {
        uw[c] = (c ? W / 2 : W) / 4;
        uh[c] = (c ? H / 2 : H) / 4;
        const size_t nu = (size_t)uw[c] * uh[c];
        if (owner[c].size() < nu) owner[c].resize(nu, 0u);
    }
    for (int b = 0; b < n_intra; b++) {
        const hevc_tu_t& t = s->tus[intra_list[(size_t)b]];
        const int c = t.c_idx, n = 1 << t.log2_size, sub = c ? 2 : 1;
        const int a = ((t.y * sub) >> p.log2_ctb) * wctb + ((t.x * sub) >> p.log2_ctb);
        ctu_of[(size_t)b] = a;
        dep_at[(size_t)b] = (int32_t)n_own;
        if (n_own + 34 > deps.size()) {
            deps.resize(deps.size() * 2);
            D = deps.data();
        }
        const size_t first_dep = n_own;
        uint32_t* own = owner[c].data();
        const int row = uw[c];
        int dp = 0;
        uint32_t last = 0;   // a run of units with one owner adds what its first unit added
        auto dep = [&](uint32_t o) {
            if ((o & GEN_BITS) != gtag || o == last) return;
            last = o;
            const int32_t ob = (int32_t)(o & 0xFFFFFFu);
            const int oa = ctu_of[(size_t)ob];
            // a CTU later in raster order is never available to this one
            // (intra_prediction.cpp:113); in tile scan one can be decoded earlier (the
            // tile to the left, below-left), and waiting for it could wait for a CTA not
            // yet started: CTAs take CTUs in raster order
            if (oa > a) return;
            for (size_t q = first_dep; q < n_own; q++)
                if (D[q] == ob) return;
            D[n_own++] = ob;
            dp = std::max(dp, level[(size_t)ob] + 1);   // local and external dependencies alike
        };
        const int ux = t.x / 4, uy = t.y / 4;
        if (t.y > 0) {
            const size_t rrow = (size_t)((t.y - 1) / 4) * row;
            const int ux0 = t.x > 0 ? (t.x - 1) / 4 : 0, ux1 = std::min(row - 1, (t.x + 2 * n - 1) / 4);
            for (int x = ux0; x <= ux1; x++) dep(own[rrow + x]);
        }
        if (t.x > 0) {
            const int lx = (t.x - 1) / 4, uy0 = t.y / 4, uy1 = std::min(uh[c] - 1, (t.y + 2 * n - 1) / 4);
            for (int y = uy0; y <= uy1; y++) dep(own[(size_t)y * row + lx]);
        }
        level[(size_t)b] = dp;
        const uint32_t mark = gtag | (uint32_t)b;
        for (int y = uy; y < uy + n / 4; y++) {
            uint32_t* r = own + (size_t)y * row;
            for (int x = ux; x < ux + n / 4; x++) r[x] = mark;
        }
    }
    dep_at[(size_t)n_intra] = (int32_t)n_own;
    deps.resize(n_own);
    // Task order: CTUs in wavefront order (key 2 * row + column, then raster), each
    // CTU's TUs by depth (every TU after the TUs it depends on, and about in the order
    // they can run), then decode order.  CTAs take CTUs by ticket in this order, so
    // the CTUs held by resident CTAs are those of the diagonal band the picture's
    // dependencies advance along (a row trails the one above by two CTUs), not whole
    // rows in raster order.  Every CTU a CTU reads from (left, above-left, above,
    // above-right) has a smaller key, so a CTA only waits for CTUs taken before its own.
    auto wave = [&](int a) { return (int64_t)(2 * (a / wctb) + a % wctb) * nctb + a; };
    auto& order = BS.order;
    order.resize((size_t)n_intra);
    bool grouped = true;   // the TUs come CTU by CTU (decode order without WPP threads)
    auto& runs = BS.runs;
    runs.clear();
    for (int b = 0; b < n_intra; b++)
        if (b == 0 || ctu_of[(size_t)b] != ctu_of[(size_t)b - 1]) runs.push_back({wave(ctu_of[(size_t)b]), b});
    {   // a CTU must form a single run: no two runs with one key
        const int nr = (int)runs.size();
        runs.push_back({INT64_MAX, n_intra});
        std::vector<std::pair<int64_t, int32_t>> sorted(runs.begin(), runs.end() - 1);
        for (int q = 0; q < nr; q++) sorted[(size_t)q].second = q;
        std::sort(sorted.begin(), sorted.end());
        for (int q = 1; q < nr && grouped; q++) grouped = sorted[(size_t)q].first != sorted[(size_t)q - 1].first;
        if (grouped) {
            auto& cnt = BS.cnt;
            int at = 0;
            for (int q = 0; q < nr; q++) {
                const int rq = sorted[(size_t)q].second;
                const int r0 = runs[(size_t)rq].second, r1 = runs[(size_t)rq + 1].second;
                int minl = level[(size_t)r0], maxl = minl;
                for (int b = r0; b < r1; b++) {
                    minl = std::min(minl, level[(size_t)b]);
                    maxl = std::max(maxl, level[(size_t)b]);
                }
                cnt.assign((size_t)(maxl - minl) + 2, 0);
                for (int b = r0; b < r1; b++) cnt[(size_t)(level[(size_t)b] - minl) + 1]++;
                for (int l = 1; l <= maxl - minl + 1; l++) cnt[(size_t)l] += cnt[(size_t)l - 1];
                for (int b = r0; b < r1; b++) order[(size_t)(at + cnt[(size_t)(level[(size_t)b] - minl)]++)] = b;
                at += r1 - r0;
            }
        }
    }
    if (!grouped) {
        for (int b = 0; b < n_intra; b++) order[(size_t)b] = b;
        std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
            const int64_t wx = wave(ctu_of[(size_t)x]), wy = wave(ctu_of[(size_t)y]);
            if (wx != wy) return wx < wy;
            return level[(size_t)x] < level[(size_t)y];
        });
    }
    auto& pos = BS.pos;   // decode order -> task order
    pos.resize((size_t)n_intra);
    itu.resize((size_t)n_intra);
    for (int i = 0; i < n_intra; i++) {
        const int b = order[(size_t)i];
        pos[(size_t)b] = i;
        itu[(size_t)i] = intra_list[(size_t)b];
        if (i == 0 || ctu_of[(size_t)b] != ctu_of[(size_t)order[(size_t)i - 1]]) {
            ictu_addr.push_back(ctu_of[(size_t)b]);
            ictu_tu_off.push_back(i);
        }
    }
    ictu_tu_off.push_back(n_intra);
    // Per CTU in task order: the task-order records (coeff_offset: the TU's offset in the
    // CTU's staged residuals; reserved[0]: ITU_PUBLISH when a TU of another CTU depends on
    // it), the residual staging entries and the dependency lists.  A dependency on a TU
    // of another CTU goes through the CTU's watcher: the distinct such TUs, in the order
    // their first dependent TU comes, each get a watch slot, and the entry names the slot
    // (INTRA_DEP_WATCH).  Earlier CTUs come first, so the records those entries mark are
    // already written.
    itu_res.assign((size_t)n_intra, make_int4(-1, 0, 0, 0));
    itu_rec.resize((size_t)n_intra);
    itu_dep.resize((size_t)n_intra);
    dep_out.resize(deps.size() + 1);   // one entry per owner found, and the spare entry
    uint32_t* dout = dep_out.data();
    uint32_t nd = 0;
    const int nic = (int)ictu_addr.size();
    auto& watch = BS.watch;
    auto& slot_of = BS.slot_of;   // (CTU index << 8) | slot of a watched TU, by task index
    watch.clear();
    ictu_watch.assign((size_t)nic, 0u);
    slot_of.assign((size_t)n_intra, -1);
    for (int k = 0; k < nic; k++) {
        int acc = 0, nw = 0;
        const uint32_t w0 = (uint32_t)watch.size();
        const int t0 = ictu_tu_off[(size_t)k], t1 = ictu_tu_off[(size_t)k + 1];
        if (t1 - t0 > IC_MAX_TUS)
            return fail(HEVCGPU_EINVAL, "CTU %d holds more intra TUs than a CTU can", ictu_addr[(size_t)k]);
        const int a = ictu_addr[(size_t)k];
        for (int i = t0; i < t1; i++) {
            const int b = order[(size_t)i];
            const hevc_tu_t& t = s->tus[itu[(size_t)i]];
            hevc_tu_t& r = itu_rec[(size_t)i];
            r = t;
            r.coeff_offset = 0;
            r.reserved[0] = 0;
            const int d0 = dep_at[(size_t)b], d1 = dep_at[(size_t)b + 1];
            itu_dep[(size_t)i] = (nd << 6) | (uint32_t)(d1 - d0);
            for (int q = d0; q < d1; q++) {
                const int ob = deps[(size_t)q], oi = pos[(size_t)ob];
                if (ctu_of[(size_t)ob] == a) {
                    dout[nd++] = (uint32_t)(oi - t0);
                    continue;
                }
                int32_t& so = slot_of[(size_t)oi];
                if (so < 0 || (so >> 8) != k) {
                    if (nw == IC_MAX_WATCH)
                        return fail(HEVCGPU_EINVAL, "CTU %d reads from more than %d intra TUs of other CTUs", a,
                                    IC_MAX_WATCH);
                    so = (k << 8) | nw++;
                    watch.push_back((uint32_t)oi);
                    itu_rec[(size_t)oi].reserved[0] = ITU_PUBLISH;
                }
                dout[nd++] = INTRA_DEP_WATCH | (uint32_t)(so & 0xFF);
            }
            if (!(t.flags & HEVC_TU_CODED)) continue;
            const int nn = 1 << (2 * t.log2_size);
            itu_res[(size_t)i] = make_int4((int)t.coeff_offset, acc, nn / 8, 0);
            r.coeff_offset = (uint32_t)acc;
            acc += nn;
        }
        if (acc > IC_MAX_RES)
            return fail(HEVCGPU_EINVAL, "CTU %d holds more intra TUs than a CTU can", a);
        ictu_watch[(size_t)k] = (w0 << 8) | (uint32_t)nw;
    }
    // one spare entry: an external dependency of task 0 on itself (the planted wait of
    // hevcgpu_job_plant_unmet_wait points task 0's list at it)
    *spare_dep = nd;
    dout[nd++] = INTRA_DEP_EXTERNAL | 0u;
    dep_out.resize(nd);
    if (dep_out.size() >= (1u << 26)) return fail(HEVCGPU_EINVAL, "intra dependency lists too long");
    return HEVCGPU_OK;
}

int job_build(hevcgpu_job* j, const hevc_picture_syntax_t* s, int stages, bool wait_uploads = true,
              bool defer = false) {
    BuildScratch& BS = t_build;
    hevcgpu_ctx* ctx = j->ctx;
    const hevc_pic_params_t& p = s->params;
    j->params = p;
    j->lay.init(p.width, p.height);
    const int W = p.width, H = p.height, gw = W / 4, gh = H / 4;
    const int ctb = 1 << p.log2_ctb;
    const int wctb = (W + ctb - 1) / ctb, hctb = (H + ctb - 1) / ctb, nctb = wctb * hctb;

    // The caller's large arrays (PUs, 4x4 grid, TUs, coefficient levels) have their own
    // device buffer and are uploaded first, so that the transfer overlaps the building of
    // the work lists below: straight from where they lie when they are in page-locked
    // memory, else through pinned staging.
    struct BigArray {
        const void* src;
        size_t bytes, off;
        bool direct;
    };
    BigArray big[4] = {{s->pus, sizeof(hevc_pu_t) * (size_t)std::max(0, s->num_pus), 0, false},
                       {s->blk, s->blk ? sizeof(uint32_t) * (size_t)gw * gh : 0, 0, false},
                       {s->tus, sizeof(hevc_tu_t) * (size_t)std::max(0, s->num_tus), 0, false},
                       {s->coeffs, sizeof(int16_t) * (size_t)s->num_coeffs, 0, false}};
    size_t big_bytes = 0;
    bool any_direct = false, any_staged = false;
    for (BigArray& b : big) {
        if (!b.src) b.bytes = 0;
        b.off = (size_t)align_up((int64_t)big_bytes, 256);
        big_bytes = b.off + b.bytes;
        b.direct = b.bytes && page_locked(b.src);
        any_direct |= b.direct;
        any_staged |= b.bytes && !b.direct;
    }
    big_bytes = std::max<size_t>(big_bytes, 256);
    int rc = j->big.get(ctx, big_bytes);
    if (rc) return rc;
    auto up = [&](const UploadOp& o) -> int {
        if (!defer) return run_upload(j, o);
        j->ops.push_back(o);
        return HEVCGPU_OK;
    };
    if (any_staged && (rc = j->pin_big.get(ctx, big_bytes))) return rc;
    // Page-locked arrays that sit in one block in this same layout (each at its offset from
    // one base, as a recorder that lays them out so puts them) go up in one copy: the gaps
    // between them are under 256 bytes, so every byte copied lies on a page that holds array
    // data.
    const uint8_t* host0 = nullptr;
    size_t first = 0, used = 0;
    bool one_block = any_direct && !any_staged;
    for (const BigArray& b : big) {
        if (!b.bytes) continue;
        const uint8_t* h = static_cast<const uint8_t*>(b.src) - b.off;
        if (!host0) {
            host0 = h;
            first = b.off;
        }
        one_block = one_block && h == host0;
        used = b.off + b.bytes;
    }
    if (one_block && host0) {
        if ((rc = up({UploadOp::COPY, static_cast<uint8_t*>(j->big.p) + first, host0 + first, used - first})))
            return rc;
    } else {
        for (const BigArray& b : big) {
            if (!b.bytes) continue;
            const void* from = b.src;
            if (!b.direct) {
                std::memcpy(static_cast<uint8_t*>(j->pin_big.p) + b.off, b.src, b.bytes);
                from = static_cast<uint8_t*>(j->pin_big.p) + b.off;
            }
            if ((rc = up({UploadOp::COPY, static_cast<uint8_t*>(j->big.p) + b.off, from, b.bytes}))) return rc;
        }
    }
    // the caller's arrays must have been read before this call returns
    if (any_direct && (rc = up({UploadOp::MARK_DIRECT, nullptr, nullptr, 0}))) return rc;

    // residual bins (coded TUs by size) and the intra TUs in decode order
    auto& bins = BS.bins;
    auto& intra_list = BS.intra_list;
    for (auto& v : bins) v.clear();
    intra_list.clear();
    for (auto& v : bins) v.reserve((size_t)s->num_tus / 2);
    intra_list.reserve((size_t)s->num_tus);
    for (int i = 0; i < s->num_tus; i++) {
        const hevc_tu_t& t = s->tus[i];
        bool intra = t.flags & HEVC_TU_INTRA;
        if ((t.flags & HEVC_TU_CODED) && (stages & (intra ? ST_INTRA : ST_RESID))) bins[t.log2_size - 2].push_back(i);
        if (intra && (stages & ST_INTRA)) intra_list.push_back(i);
    }
    j->has_intra = !intra_list.empty();
    // Intra schedule.  Per plane an owner map at 4-sample granularity records the latest
    // intra TU written there; intra TU B reads the units of its reference row
    // (x-1 .. x+2N-1 at y-1) and column (y .. y+2N-1 at x-1).  Each distinct owner is a
    // dependency of B: an owner in B's CTU a local one, an owner in an earlier CTU an
    // external one.  B's depth is one more than its deepest dependency's: the length of the
    // longest dependency chain over the picture that ends at B.  A unit whose samples B may
    // not use (availability) can only add an unneeded wait, never change a sample; owners in
    // CTUs later in raster order (decoded earlier only in tile scan) are never available
    // and add nothing.
    const int n_intra = (int)intra_list.size();
    auto& ictu_addr = BS.ictu_addr;
    auto& ictu_tu_off = BS.ictu_tu_off;
    auto& itu_rec = BS.itu_rec;         // intra TU records in task order
    auto& itu_res = BS.itu_res;         // per task entry: residual source, staged offset, 16-byte chunks
    auto& itu_dep = BS.itu_dep;         // per task entry: (dependency list offset << 6) | count
    auto& dep_out = BS.dep_out;         // dependency lists in task order
    auto& ictu_watch = BS.ictu_watch;   // per CTU: (offset in watch << 8) | count
    if ((rc = build_intra_schedule(BS, s, &j->spare_dep))) return rc;
    j->n_ictu = (int32_t)ictu_addr.size();
    // MC strips (build_mc_strips)
    auto& mc = BS.mc;
    if (stages & ST_MC) build_mc_strips(BS, s, j->lay.pitch_y, j->lay.pitch_c);
    else {
        mc[0].clear();
        mc[1].clear();
    }
    j->n_pus = s->num_pus;

    size_t o_wp, o_sao, o_sl, o_ti, o_slices, o_res[4], o_mc[2], o_ia, o_idp, o_ito, o_itu, o_iro, o_dl, o_iw, o_wl;
    size_t o_scal = 0;
    hevc_slice_t dflt{0, 0, 0, 1};
    const bool scaled = s->scaling && (stages & (ST_RESID | ST_INTRA));
    auto pack = [&](Packer& pk) {
        if (scaled) o_scal = pk.add(s->scaling, sizeof(hevc_scaling_t));
        o_wp = pk.add(s->wp, sizeof(hevc_wp_t) * (size_t)std::max(0, s->num_wp));
        o_sao = pk.add(s->sao, s->sao ? sizeof(hevc_sao_t) * (size_t)nctb : 0);
        o_sl = pk.add(s->ctb_slice, s->ctb_slice ? (size_t)nctb : 0);
        o_ti = pk.add(s->ctb_tile, s->ctb_tile ? sizeof(uint16_t) * (size_t)nctb : 0);
        o_slices = s->num_slices > 0 && s->slices ? pk.add(s->slices, sizeof(hevc_slice_t) * (size_t)s->num_slices)
                                                  : pk.add(&dflt, sizeof(dflt));
        for (int k = 0; k < 4; k++) o_res[k] = pk.add(bins[k].data(), sizeof(int32_t) * bins[k].size());
        for (int c = 0; c < 2; c++) o_mc[c] = pk.add(mc[c].data(), sizeof(uint32_t) * mc[c].size());
        o_ia = pk.add(ictu_addr.data(), sizeof(int32_t) * ictu_addr.size());
        o_ito = pk.add(ictu_tu_off.data(), sizeof(int32_t) * ictu_tu_off.size());
        o_itu = pk.add(itu_rec.data(), sizeof(hevc_tu_t) * itu_rec.size());
        o_iro = pk.add(itu_res.data(), sizeof(int4) * itu_res.size());
        o_idp = pk.add(itu_dep.data(), sizeof(uint32_t) * itu_dep.size());
        o_dl = pk.add(dep_out.data(), sizeof(uint32_t) * dep_out.size());
        o_iw = pk.add(ictu_watch.data(), sizeof(uint32_t) * ictu_watch.size());
        o_wl = pk.add(BS.watch.data(), sizeof(uint32_t) * BS.watch.size());
    };
    Packer measure;
    pack(measure);
    const size_t img = std::max<size_t>(measure.size, 256);
    j->desc_off = (size_t)align_up((int64_t)img, 256);
    if ((rc = j->recs.get(ctx, img))) return rc;
    if ((rc = j->pin.get(ctx, j->desc_off + sizeof(PicDesc)))) return rc;
    Packer write;
    write.out = static_cast<uint8_t*>(j->pin.p);
    pack(write);
    if ((rc = up({UploadOp::COPY, j->recs.p, j->pin.p, img}))) return rc;
    j->upload_bytes = big_bytes + img + sizeof(PicDesc);
    uint8_t* big_base = static_cast<uint8_t*>(j->big.p);
    uint8_t* base = static_cast<uint8_t*>(j->recs.p);

    size_t resid_bytes = j->has_intra ? sizeof(int16_t) * (size_t)align_up((int64_t)s->num_coeffs, 128) : 0;
    size_t mot_bytes = (stages & ST_DEBLOCK) ? sizeof(MotionEnt) * (size_t)align_up((int64_t)gw * gh, 32) : 0;
    size_t done_bytes = sizeof(int32_t) * (size_t)n_intra;
    rc = j->scratch.get(ctx, std::max<size_t>(resid_bytes + mot_bytes + done_bytes, 256));
    if (rc) return rc;
    rc = j->desc.get(ctx, sizeof(PicDesc));
    if (rc) return rc;

    PicDesc& D = j->host_desc;
    std::memset(&D, 0, sizeof(D));
    D.width = W;
    D.height = H;
    D.pitch_y = j->lay.pitch_y;
    D.pitch_c = j->lay.pitch_c;
    D.off_cb = j->lay.off_cb;
    D.off_cr = j->lay.off_cr;
    for (int l = 0; l < 2; l++) {
        D.num_ref[l] = p.num_ref[l];
        for (int i = 0; i < 16; i++) D.ref_poc[l][i] = p.ref_poc[l][i];
    }
    D.tus = reinterpret_cast<const hevc_tu_t*>(big_base + big[2].off);
    D.coeffs = reinterpret_cast<const int16_t*>(big_base + big[3].off);
    D.resid = resid_bytes ? static_cast<int16_t*>(j->scratch.p) : nullptr;
    D.pus = reinterpret_cast<const hevc_pu_t*>(big_base + big[0].off);
    D.wp = reinterpret_cast<const hevc_wp_t*>(base + o_wp);
    D.blk = s->blk ? reinterpret_cast<const uint32_t*>(big_base + big[1].off) : nullptr;
    D.mot = mot_bytes ? reinterpret_cast<MotionEnt*>(static_cast<uint8_t*>(j->scratch.p) + resid_bytes) : nullptr;
    D.sao = s->sao ? reinterpret_cast<const hevc_sao_t*>(base + o_sao) : nullptr;
    D.ctb_slice = s->ctb_slice ? base + o_sl : nullptr;
    D.ctb_tile = (s->ctb_tile && p.tiles_enabled) ? reinterpret_cast<const uint16_t*>(base + o_ti) : nullptr;
    D.slices = reinterpret_cast<const hevc_slice_t*>(base + o_slices);
    D.scaling = scaled ? reinterpret_cast<const hevc_scaling_t*>(base + o_scal) : nullptr;
    D.ictu_addr = reinterpret_cast<const int32_t*>(base + o_ia);
    D.ictu_tu_off = reinterpret_cast<const int32_t*>(base + o_ito);
    D.itu_rec = reinterpret_cast<const hevc_tu_t*>(base + o_itu);
    D.itu_res = reinterpret_cast<const int4*>(base + o_iro);
    D.itu_dep = reinterpret_cast<const uint32_t*>(base + o_idp);
    D.dep_list = reinterpret_cast<const uint32_t*>(base + o_dl);
    D.ictu_watch = reinterpret_cast<const uint32_t*>(base + o_iw);
    D.watch = reinterpret_cast<const uint32_t*>(base + o_wl);
    D.itu_done = reinterpret_cast<int32_t*>(static_cast<uint8_t*>(j->scratch.p) + resid_bytes + mot_bytes);
    D.n_ictu = (int32_t)ictu_addr.size();
    D.n_itu = n_intra;
    // completion flags start below every epoch a launch can use
    if (done_bytes && (rc = up({UploadOp::ZERO, D.itu_done, nullptr, done_bytes}))) return rc;
    D.num_pus = s->num_pus;
    D.num_slices = std::max(1, (int)s->num_slices);
    D.log2_ctb = p.log2_ctb;
    D.wctb = wctb;
    D.hctb = hctb;
    D.sao_enabled = p.sao_enabled && s->sao ? 1 : 0;
    D.pcm_lf_disabled = p.pcm_loop_filter_disabled;
    D.strong_intra = p.strong_intra_smoothing;
    D.intra_smoothing_disabled = p.intra_smoothing_disabled;
    D.cb_qp_offset = p.cb_qp_offset;
    D.cr_qp_offset = p.cr_qp_offset;
    D.tiles_check = (p.tiles_enabled && !p.loop_filter_across_tiles && s->ctb_tile) ? 1 : 0;
    bool multi = false;
    if (s->ctb_slice)
        for (int a = 1; a < nctb && !multi; a++) multi = s->ctb_slice[a] != s->ctb_slice[0];
    D.slice_check = multi ? 1 : 0;
    bool pcm_bypass = false;
    if (s->blk) {   // an OR over chunks of the grid (which the compiler vectorises), stopping at the first hit
        const size_t nu = (size_t)gw * gh;
        for (size_t i0 = 0; i0 < nu && !pcm_bypass; i0 += 4096) {
            const size_t i1 = std::min(nu, i0 + 4096);
            uint32_t any = 0;
            for (size_t i = i0; i < i1; i++) any |= s->blk[i];
            pcm_bypass = (any & (HEVC_BLK_PCM | HEVC_BLK_BYPASS)) != 0;
        }
    }
    D.pcm_bypass_any = pcm_bypass ? 1 : 0;
    for (int k = 0; k < 4; k++) {
        j->n_res[k] = (int32_t)bins[k].size();
        j->d_res[k] = reinterpret_cast<const int32_t*>(base + o_res[k]);
    }
    for (int c = 0; c < 2; c++) {
        j->n_mc[c] = (int32_t)mc[c].size();
        j->d_mc[c] = reinterpret_cast<const uint32_t*>(base + o_mc[c]);
    }
    // the caller may change its arrays once this returns: the direct uploads must have read
    // them, unless the caller waits for that itself (hevcgpu_job_wait_uploaded)
    if (!defer && any_direct && wait_uploads) CUDA_TRY(cudaEventSynchronize(j->direct_read));
    return HEVCGPU_OK;
}

// Point the job at its output and reference pictures and upload the descriptor.
int job_bind(hevcgpu_job* j, uint8_t* rec, uint8_t* dst, const uint8_t* const refs[2][16],
             cudaStream_t stream = nullptr) {
    if (!stream) stream = j->ctx->stream;
    PicDesc& D = j->host_desc;
    D.rec = rec;
    D.dst = dst;
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < 16; i++) D.ref[l][i] = refs ? refs[l][i] : nullptr;
    // the pinned staging copy may be rewritten only after its previous upload ran
    if (j->desc_copied) {
        CUDA_TRY(cudaEventSynchronize(j->desc_copied));
    } else {
        CUDA_TRY(cudaEventCreateWithFlags(&j->desc_copied, cudaEventDisableTiming));
    }
    uint8_t* stage = static_cast<uint8_t*>(j->pin.p) + j->desc_off;
    std::memcpy(stage, &D, sizeof(PicDesc));
    CUDA_TRY(cudaMemcpyAsync(j->desc.p, stage, sizeof(PicDesc), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaEventRecord(j->desc_copied, stream));
    return HEVCGPU_OK;
}

// ---------------------------------------------------------------------------------------
// launch sequencing over a batch of jobs
// ---------------------------------------------------------------------------------------
struct Launcher {
    hevcgpu_ctx* ctx;
    cudaStream_t s;

    template <typename K, typename... A>
    int go(K kernel, dim3 grid, dim3 block, A... args) {
        if (grid.x == 0 || grid.y == 0 || grid.z == 0) return HEVCGPU_OK;
        kernel<<<grid, block, 0, s>>>(args...);
        ctx->launches++;
        CUDA_TRY(cudaGetLastError());
        return HEVCGPU_OK;
    }

    // item-list launch over jobs[0..n): items_of(j) -> (ptr, count); per_block items per CTA
    template <typename K, typename F, typename... A>
    int items(K kernel, hevcgpu_job* const* jobs, int n, int per_block, int threads, F items_of, A... extra) {
        for (int b0 = 0; b0 < n; b0 += MAX_SEGS) {
            SegTable t;
            std::memset(&t, 0, sizeof(t));
            int blocks = 0;
            for (int k = b0; k < std::min(n, b0 + MAX_SEGS); k++) {
                const void* ptr;
                int cnt;
                items_of(jobs[k], ptr, cnt);
                if (cnt <= 0) continue;
                Seg& sg = t.s[t.n++];
                sg.items = ptr;
                sg.pic = static_cast<const PicDesc*>(jobs[k]->desc.p);
                sg.n_items = cnt;
                sg.block0 = blocks;
                blocks += (cnt + per_block - 1) / per_block;
            }
            if (t.n == 0) continue;
            int rc = go(kernel, dim3(blocks), dim3(threads), t, extra...);
            if (rc) return rc;
        }
        return HEVCGPU_OK;
    }

    // per-picture launch: grid.y = picture; grid.x from blocks_of(job)
    template <typename K, typename F>
    int pictures(K kernel, hevcgpu_job* const* jobs, int n, int threads, int z, F blocks_of) {
        for (int b0 = 0; b0 < n; b0 += MAX_SEGS) {
            SegTable t;
            std::memset(&t, 0, sizeof(t));
            int bx = 0;
            for (int k = b0; k < std::min(n, b0 + MAX_SEGS); k++) {
                Seg& sg = t.s[t.n++];
                sg.pic = static_cast<const PicDesc*>(jobs[k]->desc.p);
                bx = std::max(bx, blocks_of(jobs[k]));
            }
            int rc = go(kernel, dim3(bx, t.n, z), dim3(threads), t);
            if (rc) return rc;
        }
        return HEVCGPU_OK;
    }
};

// Brackets one stage with profiling events when profiling is on.
struct StageMark {
    hevcgpu_ctx* ctx;
    cudaStream_t stream;
    int stage;
    cudaEvent_t a = nullptr;
    uint64_t l0 = 0;
    StageMark(hevcgpu_ctx* c, cudaStream_t st, int s) : ctx(c), stream(st), stage(s) {
        if (!ctx->profiling) return;
        a = ctx->next_event();
        l0 = ctx->launches;
        if (a) cudaEventRecord(a, stream);
    }
    ~StageMark() {
        if (!ctx->profiling || !a) return;
        cudaEvent_t b = ctx->next_event();
        if (!b) return;
        cudaEventRecord(b, stream);
        ctx->marks.push_back({stage, a, b, ctx->launches - l0});
    }
};

// Where a batch runs: a CUDA stream and the flow area of its intra tasks (FlowState,
// status word, per-picture tickets).  The context's own, or a lane's.
struct Exec {
    cudaStream_t stream;
    void* flow;
    int32_t* tickets() const { return reinterpret_cast<int32_t*>(static_cast<uint8_t*>(flow) + sizeof(FlowState) + 16); }
};

int run_stages(hevcgpu_ctx* ctx, const Exec& ex, hevcgpu_job* const* jobs, int n, int stages, int res_mode) {
    Launcher L{ctx, ex.stream};
    int rc;
    if ((stages & ST_DEBLOCK) && !(stages & ST_MC)) {   // with MC, its luma strips write the grid
        StageMark m(ctx, ex.stream, 0);
        rc = L.pictures(k_motion_grid, jobs, n, 256, 1, [](hevcgpu_job* j) { return (j->n_pus * 32 + 255) / 256; });
        if (rc) return rc;
    }
    if (stages & ST_MC) {
        StageMark m(ctx, ex.stream, 1);
        rc = L.items(k_mc<false>, jobs, n, MC_THREADS, MC_THREADS, [](hevcgpu_job* j, const void*& p, int& c) {
            p = j->d_mc[0];
            c = j->n_mc[0];
        });
        if (rc) return rc;
        rc = L.items(k_mc<true>, jobs, n, MC_THREADS, MC_THREADS, [](hevcgpu_job* j, const void*& p, int& c) {
            p = j->d_mc[1];
            c = j->n_mc[1];
        });
        if (rc) return rc;
    }
    if (stages & (ST_RESID | ST_INTRA)) {
        StageMark m(ctx, ex.stream, 2);
        void (*kr[4])(const SegTable, int) = {k_residual<2>, k_residual<3>, k_residual<4>, k_residual<5>};
        for (int k = 0; k < 4; k++) {
            rc = L.items(kr[k], jobs, n, 128 >> (k + 2), 128,
                         [k](hevcgpu_job* j, const void*& p, int& c) {
                             p = j->d_res[k];
                             c = j->n_res[k];
                         },
                         res_mode);
            if (rc) return rc;
        }
    }
    if (stages & ST_INTRA) {
        StageMark m(ctx, ex.stream, 3);
        // one launch per group of up to MAX_SEGS pictures: CTAs take intra CTUs by ticket
        // in (picture, raster) order; aux0 = intra CTUs of earlier pictures, aux1 = epoch
        int k = 0;
        while (k < n) {
            SegTable t;
            std::memset(&t, 0, sizeof(t));
            int total = 0;
            for (; k < n && t.n < MAX_SEGS; k++) {
                hevcgpu_job* j = jobs[k];
                if (j->n_ictu == 0) continue;
                Seg& sg = t.s[t.n++];
                sg.pic = static_cast<const PicDesc*>(j->desc.p);
                sg.aux0 = total;
                // completion flags hold the epoch of the launch that set them; restart the
                // epochs from zero flags before they would reach the sign bit
                if (j->epoch >= 0x7FFFFFF0) {
                    CUDA_TRY(cudaMemsetAsync(j->host_desc.itu_done, 0, sizeof(int32_t) * (size_t)j->host_desc.n_itu,
                                             ex.stream));
                    j->epoch = 0;
                }
                sg.aux1 = ++j->epoch;
                total += j->n_ictu;
            }
            if (t.n == 0) continue;
            FlowState* fs = static_cast<FlowState*>(ex.flow);
            uint32_t* sticky = reinterpret_cast<uint32_t*>(fs + 1);
            int32_t* tickets = ex.tickets();
            CUDA_TRY(cudaMemsetAsync(tickets, 0, sizeof(int32_t) * (size_t)t.n, ex.stream));
            rc = L.go(k_intra_ctus, dim3(total), dim3(IC_THREADS), t, tickets, total, sticky);
            if (rc) return rc;
        }
    }
    if (stages & ST_DEBLOCK) {
        {
            StageMark m(ctx, ex.stream, 4);
            rc = L.pictures(k_deblock<true>, jobs, n, 256, 1, [](hevcgpu_job* j) {
                int segs = ((j->params.width + 7) / 8) * (j->params.height / 4);
                return (segs + 255) / 256;
            });
            if (rc) return rc;
        }
        StageMark m(ctx, ex.stream, 5);
        rc = L.pictures(k_deblock<false>, jobs, n, 256, 1, [](hevcgpu_job* j) {
            int segs = (j->params.width / 4) * ((j->params.height + 7) / 8);
            return (segs + 255) / 256;
        });
        if (rc) return rc;
    }
    if (stages & ST_SAO) {
        StageMark m(ctx, ex.stream, 6);
        // one CTA per CTB; z = 0 luma, z = 1 both chroma planes
        rc = L.pictures(k_sao, jobs, n, 256, 2, [](hevcgpu_job* j) {
            const int ctb = 1 << j->params.log2_ctb;
            return ((j->params.width + ctb - 1) / ctb) * ((j->params.height + ctb - 1) / ctb);
        });
        if (rc) return rc;
    }
    return HEVCGPU_OK;
}

int run_stages(hevcgpu_ctx* ctx, hevcgpu_job* const* jobs, int n, int stages, int res_mode) {
    return run_stages(ctx, Exec{ctx->stream, ctx->flow}, jobs, n, stages, res_mode);
}

// Copies between a pitched slot and a packed I420 host frame.  When the pitches equal the
// plane widths (widths that are multiples of 128) the slot is the packed frame itself and
// one linear copy moves it: the DMA engines run 2-D copies of many short rows well below
// the rate of a linear copy.
bool packed_layout(const Layout& L) {
    return L.pitch_y == L.W && L.pitch_c == L.W / 2 && L.off_cb == (int64_t)L.W * L.H &&
           L.off_cr == L.off_cb + (int64_t)(L.W / 2) * (L.H / 2);
}

int copy_i420(const Layout& L, uint8_t* dev, uint8_t* host, cudaMemcpyKind kind, cudaStream_t stream) {
    const int W = L.W, H = L.H, cw = W / 2, ch = H / 2;
    const bool up = kind == cudaMemcpyHostToDevice;
    if (packed_layout(L)) {
        const size_t n = (size_t)W * H + 2 * (size_t)cw * ch;
        CUDA_TRY(up ? cudaMemcpyAsync(dev, host, n, kind, stream) : cudaMemcpyAsync(host, dev, n, kind, stream));
        return HEVCGPU_OK;
    }
    uint8_t* d[3] = {dev, dev + L.off_cb, dev + L.off_cr};
    uint8_t* h[3] = {host, host + (size_t)W * H, host + (size_t)W * H + (size_t)cw * ch};
    const int w[3] = {W, cw, cw}, rows[3] = {H, ch, ch}, pitch[3] = {L.pitch_y, L.pitch_c, L.pitch_c};
    for (int p = 0; p < 3; p++)
        CUDA_TRY(up ? cudaMemcpy2DAsync(d[p], pitch[p], h[p], w[p], w[p], rows[p], kind, stream)
                    : cudaMemcpy2DAsync(h[p], w[p], d[p], pitch[p], w[p], rows[p], kind, stream));
    return HEVCGPU_OK;
}

int upload_i420(hevcgpu_ctx* ctx, const Layout& L, uint8_t* dev, const uint8_t* host) {
    return copy_i420(L, dev, const_cast<uint8_t*>(host), cudaMemcpyHostToDevice, ctx->stream);
}

int download_i420(hevcgpu_ctx* ctx, const Layout& L, const uint8_t* dev, uint8_t* host,
                  cudaStream_t stream = nullptr) {
    return copy_i420(L, const_cast<uint8_t*>(dev), host, cudaMemcpyDeviceToHost, stream ? stream : ctx->stream);
}

int check_ctx(hevcgpu_ctx* ctx) {
    if (!ctx) return fail(HEVCGPU_EINVAL, "null context");
    CUDA_TRY(cudaSetDevice(ctx->device));
    return HEVCGPU_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
extern "C" {

int hevcgpu_abi_version(void) { return HEVCGPU_ABI_VERSION; }
const char* hevcgpu_last_error(void) { return g_err.c_str(); }

int hevcgpu_create(int device, hevcgpu_ctx_t** out) {
    if (!out) return fail(HEVCGPU_EINVAL, "null out");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= device || device < 0)
        return fail(HEVCGPU_ECUDA, "no CUDA device %d (%s)", device, e != cudaSuccess ? cudaGetErrorString(e) : "count");
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(HEVCGPU_EUNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a", device,
                    prop.major, prop.minor);
    CUDA_TRY(cudaSetDevice(device));
    auto* c = new (std::nothrow) hevcgpu_ctx();
    if (!c) return fail(HEVCGPU_ENOMEM, "host allocation");
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->flow, hevcgpu_ctx::FLOW_BYTES);
    if (e == cudaSuccess) e = cudaMemset(c->flow, 0, hevcgpu_ctx::FLOW_BYTES);
    for (int k = 0; k < hevcgpu_ctx::EVENT_RING && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&c->done[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete c;
        return fail(HEVCGPU_ECUDA, "context set-up: %s", cudaGetErrorString(e));
    }
    *out = c;
    return HEVCGPU_OK;
}

void hevcgpu_destroy(hevcgpu_ctx_t* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

int hevcgpu_sync(hevcgpu_ctx_t* ctx) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return ctx->take_status();
}

void* hevcgpu_cuda_stream(hevcgpu_ctx_t* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
uint64_t hevcgpu_launch_count(hevcgpu_ctx_t* ctx) { return ctx ? ctx->launches : 0; }

int hevcgpu_set_budget(hevcgpu_ctx_t* ctx, uint64_t bytes) {
    if (!ctx) return fail(HEVCGPU_EINVAL, "null context");
    ctx->budget = bytes ? bytes : ~0ull;
    return HEVCGPU_OK;
}
uint64_t hevcgpu_bytes_in_use(hevcgpu_ctx_t* ctx) { return ctx ? ctx->allocated : 0; }

// ---- stage entry points -------------------------------------------------------------

int hevcgpu_residual_blocks(hevcgpu_ctx_t* ctx, const hevc_tu_t* tus, int32_t num_tus, const int16_t* coeffs,
                            uint64_t num_coeffs, const uint8_t* pred, uint8_t* out) {
    return hevcgpu_residual_blocks_scaled(ctx, nullptr, tus, num_tus, coeffs, num_coeffs, pred, out);
}

int hevcgpu_residual_blocks_scaled(hevcgpu_ctx_t* ctx, const hevc_scaling_t* scaling, const hevc_tu_t* tus,
                                   int32_t num_tus, const int16_t* coeffs, uint64_t num_coeffs,
                                   const uint8_t* pred, uint8_t* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (num_tus < 0 || (num_tus && (!tus || !coeffs || !pred || !out)))
        return fail(HEVCGPU_EINVAL, "null arrays");
    if (num_tus == 0) return HEVCGPU_OK;
    for (int i = 0; i < num_tus; i++) {
        const hevc_tu_t& t = tus[i];
        int n = 1 << t.log2_size;
        if (t.log2_size < 2 || t.log2_size > 5 || t.c_idx > 2 || (t.coeff_offset & 15) ||
            (uint64_t)t.coeff_offset + (uint64_t)n * n > num_coeffs || t.qp > 99)
            return fail(HEVCGPU_EINVAL, "block %d: size %d, coeff_offset %u (multiple of 16 inside the pool)", i, n,
                        t.coeff_offset);
    }
    hevcgpu_job j;
    j.ctx = ctx;
    std::vector<int32_t> bins[4];
    for (int i = 0; i < num_tus; i++) bins[tus[i].log2_size - 2].push_back(i);
    size_t o_tus, o_coef, o_pred, o_out, o_res[4], o_scal = 0;
    auto pack = [&](Packer& pk) {
        if (scaling) o_scal = pk.add(scaling, sizeof(hevc_scaling_t));
        o_tus = pk.add(tus, sizeof(hevc_tu_t) * (size_t)num_tus);
        o_coef = pk.add(coeffs, sizeof(int16_t) * (size_t)num_coeffs);
        o_pred = pk.add(pred, (size_t)num_coeffs);
        o_out = pk.add(nullptr, (size_t)num_coeffs);
        for (int k = 0; k < 4; k++) o_res[k] = pk.add(bins[k].data(), sizeof(int32_t) * bins[k].size());
    };
    Packer measure;
    pack(measure);
    const size_t img = measure.size;
    j.desc_off = (size_t)align_up((int64_t)img, 256);
    if ((rc = j.recs.get(ctx, img)) || (rc = j.desc.get(ctx, sizeof(PicDesc))) ||
        (rc = j.pin.get(ctx, j.desc_off + sizeof(PicDesc))))
        return rc;
    Packer write;
    write.out = static_cast<uint8_t*>(j.pin.p);
    pack(write);
    uint8_t* base = static_cast<uint8_t*>(j.recs.p);
    PicDesc& D = j.host_desc;
    std::memset(&D, 0, sizeof(D));
    D.tus = reinterpret_cast<const hevc_tu_t*>(base + o_tus);
    D.coeffs = reinterpret_cast<const int16_t*>(base + o_coef);
    D.rec = base + o_pred;
    D.dst = base + o_out;
    D.scaling = scaling ? reinterpret_cast<const hevc_scaling_t*>(base + o_scal) : nullptr;
    for (int k = 0; k < 4; k++) {
        j.n_res[k] = (int32_t)bins[k].size();
        j.d_res[k] = reinterpret_cast<const int32_t*>(base + o_res[k]);
    }
    CUDA_TRY(cudaMemcpyAsync(j.recs.p, j.pin.p, img, cudaMemcpyHostToDevice, ctx->stream));
    std::memcpy(static_cast<uint8_t*>(j.pin.p) + j.desc_off, &D, sizeof(D));
    CUDA_TRY(cudaMemcpyAsync(j.desc.p, static_cast<uint8_t*>(j.pin.p) + j.desc_off, sizeof(D),
                             cudaMemcpyHostToDevice, ctx->stream));
    hevcgpu_job* jp = &j;
    if ((rc = run_stages(ctx, &jp, 1, ST_RESID, RES_PACKED))) return rc;
    CUDA_TRY(cudaMemcpyAsync(out, base + o_out, (size_t)num_coeffs, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return HEVCGPU_OK;
}

}  // extern "C"

// ---- residual blocks without allocation ----------------------------------------------
// hevcgpu_residual_blocks_static runs k_residual (RES_PACKED) on caller-owned device
// buffers for callers that must not allocate while decoding: a serving process that
// sized its device memory once at start-up, and decode threads on which cudaMalloc /
// cudaFree would synchronise the device and stall the other streams' work.  Its scratch
// (picture descriptor, TU records, per-size lists of TU indices) is the fixed array
// below: one copy per device, since a __device__ variable exists in each device's
// instance of the module.  Every call writes all the scratch it reads, so nothing there
// has to start at zero.
namespace {

constexpr size_t STATIC_DESC_BYTES = 1024;
static_assert(sizeof(PicDesc) <= STATIC_DESC_BYTES, "descriptor slot of the static scratch");
static_assert(sizeof(hevc_tu_t) == 16, "TU record size");
constexpr size_t STATIC_TUS_OFF = STATIC_DESC_BYTES;
constexpr size_t STATIC_LISTS_OFF = STATIC_TUS_OFF + (size_t)HEVCGPU_STATIC_MAX_TUS * sizeof(hevc_tu_t);
constexpr size_t STATIC_SCRATCH_BYTES = STATIC_LISTS_OFF + (size_t)HEVCGPU_STATIC_MAX_TUS * sizeof(int32_t);

static __device__ __align__(256) uint8_t g_static_scratch[STATIC_SCRATCH_BYTES];

// Host side, per device: a lock that serialises whole calls (every call on a device
// shares that device's scratch array), the scratch address looked up by the device's
// first call, and the static array the per-size lists are built in.  Calls on different
// devices run side by side.
constexpr int STATIC_MAX_DEVICES = 16;
struct StaticDevice {
    std::mutex mu;
    uint8_t* base = nullptr;
    int32_t lists[HEVCGPU_STATIC_MAX_TUS];
};
StaticDevice g_static[STATIC_MAX_DEVICES];

// Waits for the calling stream when it goes out of scope, so that a call leaving early
// after queuing copies or kernels still releases its device's lock only once they are done
// with the scratch.
struct SyncOnExit {
    cudaStream_t stream;
    ~SyncOnExit() { cudaStreamSynchronize(stream); }
};

// The buffer must be device (or managed) memory of this device.
int check_device_buffer(const void* p, int device, const char* what) {
    if (reinterpret_cast<uintptr_t>(p) & 15) return fail(HEVCGPU_EINVAL, "%s is not 16-byte aligned", what);
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HEVCGPU_EINVAL, "%s: %s", what, cudaGetErrorString(e));
    }
    if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != device)
        return fail(HEVCGPU_EINVAL, "%s is not device memory of device %d", what, device);
    return HEVCGPU_OK;
}

}  // namespace

extern "C" {

int hevcgpu_residual_blocks_static(hevcgpu_ctx_t* ctx, const hevc_tu_t* tus, int32_t num_tus,
                                   const int16_t* d_coeffs, uint64_t num_coeffs, const uint8_t* d_pred,
                                   uint8_t* d_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (num_tus < 0 || (num_tus && !tus)) return fail(HEVCGPU_EINVAL, "null arrays");
    if (num_tus > HEVCGPU_STATIC_MAX_TUS)
        return fail(HEVCGPU_EINVAL, "%d blocks: the static scratch holds at most %d", num_tus,
                    HEVCGPU_STATIC_MAX_TUS);
    if (ctx->device < 0 || ctx->device >= STATIC_MAX_DEVICES)
        return fail(HEVCGPU_EUNSUPPORTED, "device %d: static scratch is kept for devices 0..%d", ctx->device,
                    STATIC_MAX_DEVICES - 1);
    if (num_tus == 0) return HEVCGPU_OK;
    if ((rc = check_device_buffer(d_coeffs, ctx->device, "levels")) ||
        (rc = check_device_buffer(d_pred, ctx->device, "prediction")) ||
        (rc = check_device_buffer(d_out, ctx->device, "output")))
        return rc;
    for (int i = 0; i < num_tus; i++) {
        const hevc_tu_t& t = tus[i];
        int n = 1 << t.log2_size;
        if (t.log2_size < 2 || t.log2_size > 5 || t.c_idx > 2 || (t.coeff_offset & 15) ||
            (uint64_t)t.coeff_offset + (uint64_t)n * n > num_coeffs || t.qp > 99)
            return fail(HEVCGPU_EINVAL, "block %d: size %d, coeff_offset %u (multiple of 16 inside the pool)", i, n,
                        t.coeff_offset);
    }

    StaticDevice& sd = g_static[ctx->device];
    std::lock_guard<std::mutex> lock(sd.mu);
    uint8_t*& base = sd.base;
    if (!base) {
        // first call on this device (its device is current): look up the scratch address
        void* p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_static_scratch));
        base = static_cast<uint8_t*>(p);
    }
    const SyncOnExit drained{ctx->stream};   // declared after the lock: runs before it is released

    // per-size lists of TU indices, back to back in the device's list array
    int32_t count[4] = {0, 0, 0, 0}, start[4];
    for (int i = 0; i < num_tus; i++) count[tus[i].log2_size - 2]++;
    start[0] = 0;
    for (int k = 1; k < 4; k++) start[k] = start[k - 1] + count[k - 1];
    int32_t fill[4] = {start[0], start[1], start[2], start[3]};
    for (int i = 0; i < num_tus; i++) sd.lists[fill[tus[i].log2_size - 2]++] = i;

    PicDesc D;
    std::memset(&D, 0, sizeof(D));
    D.tus = reinterpret_cast<const hevc_tu_t*>(base + STATIC_TUS_OFF);
    D.coeffs = d_coeffs;
    D.rec = const_cast<uint8_t*>(d_pred);  // RES_PACKED reads the prediction through rec
    D.dst = d_out;
    // pageable sources: each copy has consumed its host buffer when the call returns
    CUDA_TRY(cudaMemcpyAsync(base, &D, sizeof(D), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(base + STATIC_TUS_OFF, tus, sizeof(hevc_tu_t) * (size_t)num_tus,
                             cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(base + STATIC_LISTS_OFF, sd.lists, sizeof(int32_t) * (size_t)num_tus,
                             cudaMemcpyHostToDevice, ctx->stream));

    Launcher L{ctx, ctx->stream};
    void (*kr[4])(const SegTable, int) = {k_residual<2>, k_residual<3>, k_residual<4>, k_residual<5>};
    for (int k = 0; k < 4; k++) {
        if (count[k] == 0) continue;
        const int per_block = 128 >> (k + 2);
        SegTable t;
        std::memset(&t, 0, sizeof(t));
        t.n = 1;
        t.s[0].items = base + STATIC_LISTS_OFF + sizeof(int32_t) * (size_t)start[k];
        t.s[0].pic = reinterpret_cast<const PicDesc*>(base);
        t.s[0].n_items = count[k];
        t.s[0].block0 = 0;
        if ((rc = L.go(kr[k], dim3((count[k] + per_block - 1) / per_block), dim3(128), t, (int)RES_PACKED)))
            return rc;
    }
    // the lock is held until the kernels are done with the scratch (and `drained` waits
    // again on the way out of every earlier return)
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return HEVCGPU_OK;
}

}  // extern "C"

extern "C" {

namespace {

// Shared body of the picture-level stage entry points on host memory.
int run_host_picture(hevcgpu_ctx* ctx, const hevc_picture_syntax_t* syn, int stages, const uint8_t* in,
                     const uint8_t* const* refs, int num_refs, uint8_t* out) {
    hevcgpu_job j;
    j.ctx = ctx;
    int rc = job_build(&j, syn, stages);
    if (rc) return rc;
    const Layout& L = j.lay;
    std::vector<DevBuf> ref_bufs((size_t)std::max(0, num_refs));
    const uint8_t* ref_ptrs[2][16] = {};
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < syn->params.num_ref[l]; i++) {
            int slot = syn->params.ref_slot[l][i];
            if (!(stages & ST_MC)) continue;
            if (slot < 0 || slot >= num_refs || !refs || !refs[slot])
                return fail(HEVCGPU_EINVAL, "reference list %d entry %d names slot %d (have %d)", l, i, slot, num_refs);
            DevBuf& b = ref_bufs[(size_t)slot];
            if (!b.p) {
                if ((rc = b.get(ctx, (size_t)L.bytes))) return rc;
                if ((rc = upload_i420(ctx, L, static_cast<uint8_t*>(b.p), refs[slot]))) return rc;
            }
            ref_ptrs[l][i] = static_cast<const uint8_t*>(b.p);
        }
    DevBuf dst;
    if ((rc = j.rec.get(ctx, (size_t)L.bytes)) || (rc = dst.get(ctx, (size_t)L.bytes))) return rc;
    if (in) {
        if ((rc = upload_i420(ctx, L, static_cast<uint8_t*>(j.rec.p), in))) return rc;
    } else {
        CUDA_TRY(cudaMemsetAsync(j.rec.p, 0, (size_t)L.bytes, ctx->stream));
    }
    if ((rc = job_bind(&j, static_cast<uint8_t*>(j.rec.p), static_cast<uint8_t*>(dst.p), ref_ptrs))) return rc;
    hevcgpu_job* jp = &j;
    if ((rc = run_stages(ctx, &jp, 1, stages, RES_PICTURE))) return rc;
    const uint8_t* result = (stages & ST_SAO) ? static_cast<uint8_t*>(dst.p) : static_cast<uint8_t*>(j.rec.p);
    if ((rc = download_i420(ctx, L, result, out))) return rc;
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return ctx->take_status();
}

}  // namespace

int hevcgpu_inter_pred(hevcgpu_ctx_t* ctx, const hevc_pic_params_t* params, const hevc_pu_t* pus, int32_t num_pus,
                       const hevc_wp_t* wp, int32_t num_wp, const uint8_t* const* refs, int32_t num_refs,
                       uint8_t* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!params || !out) return fail(HEVCGPU_EINVAL, "null arguments");
    hevc_picture_syntax_t s;
    std::memset(&s, 0, sizeof(s));
    s.params = *params;
    s.num_pus = num_pus;
    s.pus = pus;
    s.num_wp = num_wp;
    s.wp = wp;
    if ((rc = validate(&s, false, true, false))) return rc;
    return run_host_picture(ctx, &s, ST_MC, nullptr, refs, num_refs, out);
}

int hevcgpu_loop_filter(hevcgpu_ctx_t* ctx, const hevc_picture_syntax_t* syn, const uint8_t* in, uint8_t* out,
                        int do_deblock, int do_sao) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!in || !out) return fail(HEVCGPU_EINVAL, "null planes");
    if ((rc = validate(syn, false, true, true))) return rc;
    int stages = (do_deblock ? ST_DEBLOCK : 0) | ST_SAO;
    hevc_picture_syntax_t s = *syn;
    if (!do_sao) s.params.sao_enabled = 0;  // the SAO pass then only copies
    return run_host_picture(ctx, &s, stages, in, nullptr, 0, out);
}

int hevcgpu_intra_recon(hevcgpu_ctx_t* ctx, const hevc_picture_syntax_t* syn, const uint8_t* in, uint8_t* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!in || !out) return fail(HEVCGPU_EINVAL, "null planes");
    if ((rc = validate(syn, true, false, false))) return rc;
    return run_host_picture(ctx, syn, ST_INTRA, in, nullptr, 0, out);
}

int hevcgpu_reconstruct_picture(hevcgpu_ctx_t* ctx, const hevc_picture_syntax_t* syn, const uint8_t* const* refs,
                                int32_t num_refs, uint8_t* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out) return fail(HEVCGPU_EINVAL, "null output");
    if ((rc = validate(syn, true, true, true))) return rc;
    return run_host_picture(ctx, syn, ST_ALL, nullptr, refs, num_refs, out);
}

// ---- DPB / picture pipeline ----------------------------------------------------------

int hevcgpu_stream_open(hevcgpu_ctx_t* ctx, int32_t width, int32_t height, int32_t bit_depth, int32_t num_slots,
                        hevcgpu_stream_t** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out) return fail(HEVCGPU_EINVAL, "null out");
    *out = nullptr;
    if (bit_depth != 8) return fail(HEVCGPU_EUNSUPPORTED, "bit depth %d", bit_depth);
    if (width <= 0 || height <= 0 || (width & 7) || (height & 7) || num_slots <= 0 || num_slots > 64)
        return fail(HEVCGPU_EINVAL, "stream %dx%d with %d slots", width, height, num_slots);
    auto* st = new (std::nothrow) hevcgpu_stream();
    if (!st) return fail(HEVCGPU_ENOMEM, "host allocation");
    st->ctx = ctx;
    st->lay.init(width, height);
    st->slots.resize((size_t)num_slots);
    for (auto& b : st->slots) {
        if ((rc = b.get(ctx, (size_t)st->lay.bytes))) {
            delete st;
            return rc;
        }
    }
    *out = st;
    return HEVCGPU_OK;
}

void hevcgpu_stream_close(hevcgpu_stream_t* st) {
    if (!st) return;
    cudaStreamSynchronize(st->ctx->stream);
    delete st;
}

int hevcgpu_slot_upload(hevcgpu_stream_t* st, int32_t slot, const uint8_t* i420) {
    if (!st || !i420 || slot < 0 || slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", slot);
    int rc = st->wait_slot_read(slot, st->ctx->stream);
    if (rc) return fail(rc, "waiting for the downloads of slot %d", slot);
    rc = upload_i420(st->ctx, st->lay, static_cast<uint8_t*>(st->slots[(size_t)slot].p), i420);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(st->ctx->stream));
    return HEVCGPU_OK;
}

int hevcgpu_slot_download(hevcgpu_stream_t* st, int32_t slot, uint8_t* i420) {
    if (!st || !i420 || slot < 0 || slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", slot);
    int rc = download_i420(st->ctx, st->lay, static_cast<uint8_t*>(st->slots[(size_t)slot].p), i420);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(st->ctx->stream));
    return HEVCGPU_OK;
}

int hevcgpu_slot_download_frame(hevcgpu_stream_t* st, int32_t slot, const hevc_crop_t* crop, uint16_t* y,
                                int32_t stride_y, uint16_t* cb, uint16_t* cr, int32_t stride_c) {
    if (!st || slot < 0 || slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", slot);
    if (!y || !cb || !cr) return fail(HEVCGPU_EINVAL, "null planes");
    const Layout& L = st->lay;
    const hevc_crop_t c = crop ? *crop : hevc_crop_t{0, 0, 0, 0};
    if (c.left < 0 || c.right < 0 || c.top < 0 || c.bottom < 0 || ((c.left | c.right | c.top | c.bottom) & 1) ||
        c.left + c.right >= L.W || c.top + c.bottom >= L.H)
        return fail(HEVCGPU_EINVAL, "conformance window %d,%d,%d,%d (even luma offsets inside %dx%d)", c.left, c.right,
                    c.top, c.bottom, L.W, L.H);
    const int w = L.W - c.left - c.right, h = L.H - c.top - c.bottom;
    if (stride_y < w || stride_c < w / 2) return fail(HEVCGPU_EINVAL, "strides %d/%d below %d/%d", stride_y, stride_c, w, w / 2);
    int rc = check_ctx(st->ctx);
    if (rc) return rc;
    const uint8_t* s = static_cast<const uint8_t*>(st->slots[(size_t)slot].p);
    WidenArgs a{};
    uint16_t* host[3] = {y, cb, cr};
    const int32_t host_stride[3] = {stride_y, stride_c, stride_c};
    a.src[0] = s + (int64_t)c.top * L.pitch_y + c.left;
    a.src[1] = s + L.off_cb + (int64_t)(c.top / 2) * L.pitch_c + c.left / 2;
    a.src[2] = s + L.off_cr + (int64_t)(c.top / 2) * L.pitch_c + c.left / 2;
    size_t bytes = 0, off[3];
    for (int p = 0; p < 3; p++) {
        a.src_pitch[p] = p ? L.pitch_c : L.pitch_y;
        a.w[p] = p ? w / 2 : w;
        a.h[p] = p ? h / 2 : h;
        a.vecs[p] = (a.w[p] + 7) / 8;
        a.first[p] = p ? a.first[p - 1] + (int64_t)a.vecs[p - 1] * a.h[p - 1] : 0;
        off[p] = bytes;
        bytes += (size_t)align_up((int64_t)a.vecs[p] * 16 * a.h[p], 256);
    }
    a.total = a.first[2] + (int64_t)a.vecs[2] * a.h[2];
    DevBuf stage;
    if ((rc = stage.get(st->ctx, bytes))) return rc;
    for (int p = 0; p < 3; p++) a.dst[p] = reinterpret_cast<uint16_t*>(static_cast<uint8_t*>(stage.p) + off[p]);
    const int threads = 256;
    k_widen_frame<<<(unsigned)((a.total + threads - 1) / threads), threads, 0, st->ctx->stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    for (int p = 0; p < 3; p++)
        CUDA_TRY(cudaMemcpy2DAsync(host[p], (size_t)host_stride[p] * 2, a.dst[p], (size_t)a.vecs[p] * 16,
                                   (size_t)a.w[p] * 2, (size_t)a.h[p], cudaMemcpyDeviceToHost, st->ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(st->ctx->stream));
    return HEVCGPU_OK;
}

int hevcgpu_slot_checksum(hevcgpu_stream_t* st, int32_t slot, const hevc_crop_t* crop, uint32_t* out) {
    if (!st || slot < 0 || slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", slot);
    if (!out) return fail(HEVCGPU_EINVAL, "null out");
    const Layout& L = st->lay;
    const hevc_crop_t c = crop ? *crop : hevc_crop_t{0, 0, 0, 0};
    if (c.left < 0 || c.right < 0 || c.top < 0 || c.bottom < 0 || ((c.left | c.right | c.top | c.bottom) & 1) ||
        c.left + c.right >= L.W || c.top + c.bottom >= L.H)
        return fail(HEVCGPU_EINVAL, "conformance window %d,%d,%d,%d (even luma offsets inside %dx%d)", c.left, c.right,
                    c.top, c.bottom, L.W, L.H);
    int rc = check_ctx(st->ctx);
    if (rc) return rc;
    const int w = L.W - c.left - c.right, h = L.H - c.top - c.bottom;
    const uint8_t* s = static_cast<const uint8_t*>(st->slots[(size_t)slot].p);
    ChecksumArgs a{};
    a.src[0] = s + (int64_t)c.top * L.pitch_y + c.left;
    a.src[1] = s + L.off_cb + (int64_t)(c.top / 2) * L.pitch_c + c.left / 2;
    a.src[2] = s + L.off_cr + (int64_t)(c.top / 2) * L.pitch_c + c.left / 2;
    for (int p = 0; p < 3; p++) {
        a.pitch[p] = p ? L.pitch_c : L.pitch_y;
        a.w[p] = p ? w / 2 : w;
        a.h[p] = p ? h / 2 : h;
    }
    DevBuf sums;
    if ((rc = sums.get(st->ctx, 3 * sizeof(uint32_t)))) return rc;
    a.out = static_cast<uint32_t*>(sums.p);
    CUDA_TRY(cudaMemsetAsync(a.out, 0, 3 * sizeof(uint32_t), st->ctx->stream));
    k_picture_checksum<<<dim3((unsigned)std::min(h, 2 * st->ctx->sm_count), 3), 256, 0, st->ctx->stream>>>(a);
    st->ctx->launches++;
    CUDA_TRY(cudaGetLastError());
    uint32_t host[3];
    CUDA_TRY(cudaMemcpyAsync(host, a.out, sizeof(host), cudaMemcpyDeviceToHost, st->ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(st->ctx->stream));
    for (int p = 0; p < 3; p++) out[p] = host[p];
    return HEVCGPU_OK;
}

int hevcgpu_slot_device_ptr(hevcgpu_stream_t* st, int32_t slot, void** y, void** cb, void** cr, int32_t* pitch_y,
                            int32_t* pitch_c) {
    if (!st || slot < 0 || slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", slot);
    uint8_t* b = static_cast<uint8_t*>(st->slots[(size_t)slot].p);
    if (y) *y = b;
    if (cb) *cb = b + st->lay.off_cb;
    if (cr) *cr = b + st->lay.off_cr;
    if (pitch_y) *pitch_y = st->lay.pitch_y;
    if (pitch_c) *pitch_c = st->lay.pitch_c;
    return HEVCGPU_OK;
}

namespace {
// defer: the job's CUDA calls stay queued in it for job_issue (batched preparation).
int job_prepare(hevcgpu_stream_t* st, const hevc_picture_syntax_t* syn, hevcgpu_job_t** out, bool wait_uploads,
                bool defer = false) {
    if (!st || !out) return fail(HEVCGPU_EINVAL, "null arguments");
    *out = nullptr;
    int rc = check_ctx(st->ctx);
    if (rc) return rc;
    if ((rc = validate(syn, true, true, true))) return rc;
    if (syn->params.width != st->lay.W || syn->params.height != st->lay.H)
        return fail(HEVCGPU_EINVAL, "picture %dx%d on a %dx%d stream", syn->params.width, syn->params.height,
                    st->lay.W, st->lay.H);
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < syn->params.num_ref[l]; i++) {
            int s = syn->params.ref_slot[l][i];
            if (s < 0 || s >= (int)st->slots.size())
                return fail(HEVCGPU_EINVAL, "reference list %d entry %d names slot %d", l, i, s);
        }
    auto* j = new (std::nothrow) hevcgpu_job();
    if (!j) return fail(HEVCGPU_ENOMEM, "host allocation");
    j->ctx = st->ctx;
    j->st = st;
    if ((rc = job_build(j, syn, ST_ALL, wait_uploads, defer)) || (rc = j->rec.get(st->ctx, (size_t)j->lay.bytes))) {
        delete j;
        return rc;
    }
    {
        std::lock_guard<std::mutex> g(st->ctx->jobs_mu);
        st->ctx->live_jobs.insert(j);
        j->registered = true;
    }
    *out = j;
    return HEVCGPU_OK;
}
}  // namespace

int hevcgpu_job_prepare(hevcgpu_stream_t* st, const hevc_picture_syntax_t* syn, hevcgpu_job_t** out) {
    return job_prepare(st, syn, out, true);
}

static_assert(HEVC_INTRA_DEP_WATCH == INTRA_DEP_WATCH && HEVC_INTRA_PUBLISH == ITU_PUBLISH,
              "the schedule the diagnostic hands out is the one the kernel reads");

int hevcgpu_intra_schedule(const hevc_picture_syntax_t* syn, hevc_intra_schedule_t* out) {
    if (!out) return fail(HEVCGPU_EINVAL, "null out");
    std::memset(out, 0, sizeof(*out));
    int rc = validate(syn, true, false, false);
    if (rc) return rc;
    BuildScratch& BS = t_build;
    BS.intra_list.clear();
    for (int i = 0; i < syn->num_tus; i++)
        if (syn->tus[i].flags & HEVC_TU_INTRA) BS.intra_list.push_back(i);
    uint32_t spare = 0;
    if ((rc = build_intra_schedule(BS, syn, &spare))) return rc;
    BS.task_flags.resize(BS.itu_rec.size());
    for (size_t i = 0; i < BS.itu_rec.size(); i++) BS.task_flags[i] = BS.itu_rec[i].reserved[0];
    out->n_ctu = (int32_t)BS.ictu_addr.size();
    out->n_task = (int32_t)BS.intra_list.size();
    out->n_dep = BS.intra_list.empty() ? 0 : (int32_t)spare;   // the entries before the spare one
    out->n_watch = (int32_t)BS.watch.size();
    out->ctu_addr = BS.ictu_addr.data();
    out->ctu_first = BS.ictu_tu_off.data();
    out->task_tu = BS.itu.data();
    out->task_deps = BS.itu_dep.data();
    out->deps = BS.dep_out.data();
    out->task_flags = BS.task_flags.data();
    out->ctu_watch = BS.ictu_watch.data();
    out->watch = BS.watch.data();
    return HEVCGPU_OK;
}

int hevcgpu_mc_strips(const hevc_picture_syntax_t* syn, const uint32_t** luma, int32_t* n_luma,
                      const uint32_t** chroma, int32_t* n_chroma) {
    if (!luma || !n_luma || !chroma || !n_chroma) return fail(HEVCGPU_EINVAL, "null out");
    *luma = *chroma = nullptr;
    *n_luma = *n_chroma = 0;
    int rc = validate(syn, false, true, false);
    if (rc) return rc;
    Layout lay;
    lay.init(syn->params.width, syn->params.height);
    BuildScratch& BS = t_build;
    build_mc_strips(BS, syn, lay.pitch_y, lay.pitch_c);
    *luma = BS.mc[0].data();
    *n_luma = (int32_t)BS.mc[0].size();
    *chroma = BS.mc[1].data();
    *n_chroma = (int32_t)BS.mc[1].size();
    return HEVCGPU_OK;
}

int hevcgpu_job_plant_unmet_wait(hevcgpu_job_t* job) {
    if (!job) return fail(HEVCGPU_EINVAL, "null job");
    if (job->n_ictu <= 0) return fail(HEVCGPU_EINVAL, "the job has no intra CTU to plant a wait in");
    int rc = check_ctx(job->ctx);
    if (rc) return rc;
    // Task 0 (the first TU of the first intra CTU) depends on nothing.  Its dependency list
    // now is the job's spare entry: an external dependency on its own completion, which only
    // it could publish.
    const PicDesc& D = job->host_desc;
    cudaStream_t s = job->ctx->stream;
    const uint32_t e = (job->spare_dep << 6) | 1u;
    CUDA_TRY(cudaMemcpyAsync(const_cast<uint32_t*>(D.itu_dep), &e, sizeof(e), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));   // the copy read e before it goes
    return HEVCGPU_OK;
}

int hevcgpu_job_wait_uploaded(hevcgpu_job_t* job) {
    if (!job) return fail(HEVCGPU_EINVAL, "null job");
    if (job->direct_read) CUDA_TRY(cudaEventSynchronize(job->direct_read));
    return HEVCGPU_OK;
}

uint64_t hevcgpu_job_upload_bytes(hevcgpu_job_t* job) { return job ? job->upload_bytes : 0; }

int hevcgpu_host_alloc(size_t bytes, void** out) {
    if (!out) return fail(HEVCGPU_EINVAL, "null out");
    *out = nullptr;
    if (bytes == 0) return fail(HEVCGPU_EINVAL, "zero bytes");
    if (cudaHostAlloc(out, bytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return fail(HEVCGPU_ENOMEM, "cudaHostAlloc of %zu bytes failed", bytes);
    }
    return HEVCGPU_OK;
}

int hevcgpu_host_free(void* p) {
    if (!p) return HEVCGPU_OK;
    CUDA_TRY(cudaFreeHost(p));
    return HEVCGPU_OK;
}

void hevcgpu_job_free(hevcgpu_job_t* job) {
    if (!job) return;
    delete job;   // waits for the job's own last use (see ~hevcgpu_job)
}

namespace {
// Jobs last launched on another stream: make `stream` wait for those launches (their
// descriptors and scratch are reused).
int order_jobs(hevcgpu_job* const* jobs, int n, cudaStream_t stream) {
    cudaEvent_t waited[8];
    int nw = 0;
    for (int k = 0; k < n; k++) {
        hevcgpu_job* j = jobs[k];
        if (!j->last_done || j->last_stream == stream) continue;
        bool seen = false;
        for (int q = 0; q < nw && !seen; q++) seen = waited[q] == j->last_done;
        if (seen) continue;
        CUDA_TRY(cudaStreamWaitEvent(stream, j->last_done, 0));
        if (nw < 8) waited[nw++] = j->last_done;
    }
    return HEVCGPU_OK;
}
// After a launch on `stream`: record its completion event and remember it in the jobs.
int mark_jobs(hevcgpu_job* const* jobs, int n, cudaStream_t stream, cudaEvent_t done) {
    CUDA_TRY(cudaEventRecord(done, stream));
    for (int k = 0; k < n; k++) {
        jobs[k]->last_stream = stream;
        jobs[k]->last_done = done;
    }
    return HEVCGPU_OK;
}

int job_target(hevcgpu_job* j, int32_t dst_slot, cudaStream_t stream = nullptr) {
    hevcgpu_stream* st = j->st;
    if (!st) return fail(HEVCGPU_EINVAL, "job has no stream");
    if (dst_slot < 0 || dst_slot >= (int)st->slots.size()) return fail(HEVCGPU_EINVAL, "bad slot %d", dst_slot);
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < j->params.num_ref[l]; i++)
            if (j->params.ref_slot[l][i] == dst_slot)
                return fail(HEVCGPU_EINVAL, "slot %d is both a reference and the destination", dst_slot);
    if (j->dst_slot == dst_slot) return HEVCGPU_OK;
    const uint8_t* refs[2][16] = {};
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < j->params.num_ref[l]; i++)
            refs[l][i] = static_cast<const uint8_t*>(st->slots[(size_t)j->params.ref_slot[l][i]].p);
    int rc = job_bind(j, static_cast<uint8_t*>(j->rec.p), static_cast<uint8_t*>(st->slots[(size_t)dst_slot].p), refs,
                      stream);
    if (rc) return rc;
    j->dst_slot = dst_slot;
    return HEVCGPU_OK;
}
}  // namespace

namespace {
// Checks of a batch: one context, no job twice, no two pictures into one slot of a stream.
int check_batch(hevcgpu_job_t* const* jobs, const int32_t* dst_slots, int32_t n, hevcgpu_ctx** ctx_out) {
    if (!jobs || !dst_slots || n <= 0) return fail(HEVCGPU_EINVAL, "empty batch");
    if (!jobs[0]) return fail(HEVCGPU_EINVAL, "null job");
    hevcgpu_ctx* ctx = jobs[0]->ctx;
    for (int k = 0; k < n; k++) {
        if (!jobs[k] || jobs[k]->ctx != ctx) return fail(HEVCGPU_EINVAL, "batch mixes contexts");
        for (int q = 0; q < k; q++) {
            if (jobs[q] == jobs[k]) return fail(HEVCGPU_EINVAL, "job %d appears twice in the batch", k);
            if (jobs[q]->st == jobs[k]->st && dst_slots[q] == dst_slots[k])
                return fail(HEVCGPU_EINVAL, "two pictures of the batch write slot %d of one stream", dst_slots[k]);
        }
    }
    *ctx_out = ctx;
    return HEVCGPU_OK;
}

// A batch on an execution stream: order after the jobs' launches elsewhere, point the
// jobs at their slots, run the stages, record completion.
int launch_batch(hevcgpu_ctx* ctx, const Exec& ex, cudaEvent_t done, hevcgpu_job* const* jobs,
                 const int32_t* dst_slots, int n) {
    int rc = order_jobs(jobs, n, ex.stream);
    if (rc) return rc;
    for (int k = 0; k < n; k++) {
        if (jobs[k]->st && (rc = jobs[k]->st->wait_slot_read(dst_slots[k], ex.stream)))
            return fail(rc, "waiting for the downloads of slot %d", dst_slots[k]);
        if ((rc = job_target(jobs[k], dst_slots[k], ex.stream))) return rc;
    }
    if ((rc = run_stages(ctx, ex, jobs, n, ST_ALL, RES_PICTURE))) return rc;
    return mark_jobs(jobs, n, ex.stream, done);
}
}  // namespace

int hevcgpu_job_launch(hevcgpu_job_t* job, int32_t dst_slot) {
    if (!job) return fail(HEVCGPU_EINVAL, "null job");
    hevcgpu_job* jp = job;
    return launch_batch(job->ctx, Exec{job->ctx->stream, job->ctx->flow}, job->ctx->next_done(), &jp, &dst_slot, 1);
}

int hevcgpu_batch_launch(hevcgpu_job_t* const* jobs, const int32_t* dst_slots, int32_t n) {
    hevcgpu_ctx* ctx = nullptr;
    int rc = check_batch(jobs, dst_slots, n, &ctx);
    if (rc) return rc;
    return launch_batch(ctx, Exec{ctx->stream, ctx->flow}, ctx->next_done(), jobs, dst_slots, n);
}

// ---- lanes ---------------------------------------------------------------------------

int hevcgpu_lane_open(hevcgpu_ctx_t* ctx, hevcgpu_lane_t** out) {
    if (!out) return fail(HEVCGPU_EINVAL, "null out");
    *out = nullptr;
    int rc = check_ctx(ctx);
    if (rc) return rc;
    auto* ln = new (std::nothrow) hevcgpu_lane();
    if (!ln) return fail(HEVCGPU_ENOMEM, "host allocation");
    ln->ctx = ctx;
    cudaError_t e = cudaStreamCreateWithFlags(&ln->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&ln->flow, hevcgpu_ctx::FLOW_BYTES);
    if (e == cudaSuccess) e = cudaMemset(ln->flow, 0, hevcgpu_ctx::FLOW_BYTES);
    for (int k = 0; k < hevcgpu_ctx::EVENT_RING && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&ln->done[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ln->ctx_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ln->cstream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ln->src_ready, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete ln;
        return fail(HEVCGPU_ECUDA, "lane set-up: %s", cudaGetErrorString(e));
    }
    *out = ln;
    return HEVCGPU_OK;
}

void hevcgpu_lane_close(hevcgpu_lane_t* lane) {
    if (!lane) return;
    cudaSetDevice(lane->ctx->device);
    cudaStreamSynchronize(lane->stream);
    cudaStreamSynchronize(lane->cstream);
    {   // jobs last launched on this lane forget it: its work is done
        std::lock_guard<std::mutex> g(lane->ctx->jobs_mu);
        for (hevcgpu_job* j : lane->ctx->live_jobs)
            if (j->last_stream == lane->stream) {
                j->last_stream = nullptr;
                j->last_done = nullptr;
            }
    }
    delete lane;
}

int hevcgpu_lane_batch_launch(hevcgpu_lane_t* lane, hevcgpu_job_t* const* jobs, const int32_t* dst_slots,
                              int32_t n) {
    if (!lane) return fail(HEVCGPU_EINVAL, "null lane");
    hevcgpu_ctx* ctx = nullptr;
    int rc = check_batch(jobs, dst_slots, n, &ctx);
    if (rc) return rc;
    if (ctx != lane->ctx) return fail(HEVCGPU_EINVAL, "jobs of another context");
    // the jobs' record uploads and the slots' uploads ran on the context's stream
    CUDA_TRY(cudaEventRecord(lane->ctx_ready, ctx->stream));
    CUDA_TRY(cudaStreamWaitEvent(lane->stream, lane->ctx_ready, 0));
    return launch_batch(ctx, Exec{lane->stream, lane->flow}, lane->next_done(), jobs, dst_slots, n);
}

int hevcgpu_lane_sync(hevcgpu_lane_t* lane) {
    if (!lane) return fail(HEVCGPU_EINVAL, "null lane");
    CUDA_TRY(cudaStreamSynchronize(lane->stream));
    CUDA_TRY(cudaStreamSynchronize(lane->cstream));
    return hevcgpu_ctx::take_status_of(lane->flow);
}

void* hevcgpu_lane_cuda_stream(hevcgpu_lane_t* lane) { return lane ? (void*)lane->stream : nullptr; }
void* hevcgpu_lane_copy_stream(hevcgpu_lane_t* lane) { return lane ? (void*)lane->cstream : nullptr; }

namespace {
int jobs_prepare(hevcgpu_stream_t* const* sts, const hevc_picture_syntax_t* const* syns, int32_t n,
                 hevcgpu_job_t** out, bool wait_uploads) {
    if (n < 0 || (n && (!sts || !syns || !out))) return fail(HEVCGPU_EINVAL, "null arrays");
    if (n == 0) return HEVCGPU_OK;
    for (int i = 0; i < n; i++) {
        out[i] = nullptr;
        if (!sts[i] || !syns[i]) return fail(HEVCGPU_EINVAL, "picture %d: null stream or syntax", i);
        if (sts[i]->ctx != sts[0]->ctx) return fail(HEVCGPU_EINVAL, "picture %d: streams of two contexts", i);
    }
    hevcgpu_ctx* ctx = sts[0]->ctx;
    int rc = check_ctx(ctx);
    if (rc) return rc;
    std::vector<int> rcs((size_t)n, 0);
    std::vector<std::string> msgs((size_t)n);
    {
        std::lock_guard<std::mutex> g(ctx->pool.run_mu);
        ctx->pool.ensure(ctx->device);
        // the workers build the jobs' host images; their CUDA calls are issued below, from
        // this thread, picture by picture
        ctx->pool.run(n, [&](int i) {
            rcs[(size_t)i] = job_prepare(sts[i], syns[i], &out[i], wait_uploads, true);
            if (rcs[(size_t)i]) msgs[(size_t)i] = g_err;
        });
    }
    bool built = true;
    for (int i = 0; i < n; i++) built = built && !rcs[(size_t)i];
    for (int i = 0; i < n && built; i++)
        if ((rcs[(size_t)i] = job_issue(out[i]))) {
            msgs[(size_t)i] = g_err;
            built = false;
        }
    for (int i = 0; i < n; i++) {
        if (!rcs[(size_t)i]) continue;
        for (int k = 0; k < n; k++) {
            hevcgpu_job_free(out[k]);
            out[k] = nullptr;
        }
        return fail(rcs[(size_t)i], "picture %d: %s", i, msgs[(size_t)i].c_str());
    }
    // the caller may change its arrays once this returns (unless it waits for the uploads
    // itself, hevcgpu_job_wait_uploaded)
    if (wait_uploads)
        for (int i = 0; i < n; i++)
            if (out[i]->direct_read) CUDA_TRY(cudaEventSynchronize(out[i]->direct_read));
    return HEVCGPU_OK;
}
}  // namespace

int hevcgpu_jobs_prepare(hevcgpu_stream_t* const* sts, const hevc_picture_syntax_t* const* syns, int32_t n,
                         hevcgpu_job_t** out) {
    return jobs_prepare(sts, syns, n, out, true);
}

int hevcgpu_jobs_prepare_async(hevcgpu_stream_t* const* sts, const hevc_picture_syntax_t* const* syns, int32_t n,
                               hevcgpu_job_t** out) {
    return jobs_prepare(sts, syns, n, out, false);
}

}  // extern "C"

namespace {
// Batched download with the device->host copies on `stream` (null: the context's).
int slots_download_on(hevcgpu_stream_t* const* sts, const int32_t* slots, int32_t n, uint8_t* const* outs,
                      cudaStream_t stream) {
    if (n < 0 || (n && (!sts || !slots || !outs))) return fail(HEVCGPU_EINVAL, "null arrays");
    if (n == 0) return HEVCGPU_OK;
    for (int i = 0; i < n; i++) {
        if (!sts[i] || !outs[i]) return fail(HEVCGPU_EINVAL, "picture %d: null stream or buffer", i);
        if (sts[i]->ctx != sts[0]->ctx) return fail(HEVCGPU_EINVAL, "picture %d: streams of two contexts", i);
        if (slots[i] < 0 || slots[i] >= (int)sts[i]->slots.size())
            return fail(HEVCGPU_EINVAL, "picture %d: bad slot %d", i, slots[i]);
    }
    hevcgpu_ctx* ctx = sts[0]->ctx;
    int rc = check_ctx(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(ctx->pool.run_mu);
    ctx->pool.ensure(ctx->device);
    while ((int)ctx->dl_events.size() < n) {
        cudaEvent_t e;
        CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->dl_events.push_back(e);
    }
    // Pageable buffers go through pinned staging, which the workers copy out as soon as
    // each picture's copies have landed; pinned (registered) buffers take the DMA directly.
    std::vector<HostBuf> stage((size_t)n);
    for (int i = 0; i < n; i++) {
        const Layout& L = sts[i]->lay;
        const size_t bytes = (size_t)L.W * L.H * 3 / 2;
        cudaPointerAttributes a;
        const bool pinned = cudaPointerGetAttributes(&a, outs[i]) == cudaSuccess && a.type == cudaMemoryTypeHost;
        cudaGetLastError();
        uint8_t* dst = outs[i];
        if (!pinned) {
            if ((rc = stage[(size_t)i].get(ctx, bytes))) return rc;
            dst = static_cast<uint8_t*>(stage[(size_t)i].p);
        }
        if ((rc = download_i420(ctx, L, static_cast<uint8_t*>(sts[i]->slots[(size_t)slots[i]].p), dst, stream)))
            return rc;
        CUDA_TRY(cudaEventRecord(ctx->dl_events[(size_t)i], stream ? stream : ctx->stream));
    }
    std::vector<int> rcs((size_t)n, 0);
    ctx->pool.run(n, [&](int i) {
        if (cudaEventSynchronize(ctx->dl_events[(size_t)i]) != cudaSuccess) {
            rcs[(size_t)i] = HEVCGPU_ECUDA;
            return;
        }
        if (stage[(size_t)i].p) {
            const Layout& L = sts[i]->lay;
            std::memcpy(outs[i], stage[(size_t)i].p, (size_t)L.W * L.H * 3 / 2);
        }
    });
    for (int i = 0; i < n; i++)
        if (rcs[(size_t)i]) return fail(HEVCGPU_ECUDA, "picture %d: download: %s", i, cudaGetErrorString(cudaGetLastError()));
    return HEVCGPU_OK;
}

}  // namespace

extern "C" {

int hevcgpu_slots_download(hevcgpu_stream_t* const* sts, const int32_t* slots, int32_t n, uint8_t* const* outs) {
    return slots_download_on(sts, slots, n, outs, nullptr);
}

int hevcgpu_lane_slots_download(hevcgpu_lane_t* lane, hevcgpu_stream_t* const* sts, const int32_t* slots, int32_t n,
                                uint8_t* const* outs) {
    if (!lane) return fail(HEVCGPU_EINVAL, "null lane");
    for (int i = 0; i < n; i++)
        if (sts && sts[i] && sts[i]->ctx != lane->ctx) return fail(HEVCGPU_EINVAL, "picture %d: stream of another context", i);
    int rc = slots_download_on(sts, slots, n, outs, lane->stream);
    if (rc) return rc;
    return hevcgpu_ctx::take_status_of(lane->flow);
}

int hevcgpu_lane_slots_download_async(hevcgpu_lane_t* lane, hevcgpu_stream_t* const* sts, const int32_t* slots,
                                      int32_t n, uint8_t* const* outs, uint64_t* ticket) {
    if (!lane || !ticket) return fail(HEVCGPU_EINVAL, "null lane or ticket");
    *ticket = 0;
    if (n < 0 || (n && (!sts || !slots || !outs))) return fail(HEVCGPU_EINVAL, "null arrays");
    for (int i = 0; i < n; i++) {
        if (!sts[i] || !outs[i]) return fail(HEVCGPU_EINVAL, "picture %d: null stream or buffer", i);
        if (sts[i]->ctx != lane->ctx) return fail(HEVCGPU_EINVAL, "picture %d: stream of another context", i);
        if (slots[i] < 0 || slots[i] >= (int)sts[i]->slots.size())
            return fail(HEVCGPU_EINVAL, "picture %d: bad slot %d", i, slots[i]);
        cudaPointerAttributes a;
        const bool pinned = cudaPointerGetAttributes(&a, outs[i]) == cudaSuccess && a.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (!pinned) return fail(HEVCGPU_EINVAL, "picture %d: destination is not page-locked host memory", i);
    }
    int rc = check_ctx(lane->ctx);
    if (rc) return rc;
    // the copies follow the lane's work queued so far, on the lane's copy stream
    CUDA_TRY(cudaEventRecord(lane->src_ready, lane->stream));
    CUDA_TRY(cudaStreamWaitEvent(lane->cstream, lane->src_ready, 0));
    for (int i = 0; i < n; i++)
        if ((rc = download_i420(lane->ctx, sts[i]->lay, static_cast<uint8_t*>(sts[i]->slots[(size_t)slots[i]].p),
                                outs[i], lane->cstream)))
            return rc;
    for (int i = 0; i < n; i++) {   // later writes of these slots wait for the copies
        hevcgpu_stream* st = sts[i];
        if (st->slot_read.size() < st->slots.size()) st->slot_read.resize(st->slots.size(), nullptr);
        cudaEvent_t& r = st->slot_read[(size_t)slots[i]];
        if (!r) CUDA_TRY(cudaEventCreateWithFlags(&r, cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(r, lane->cstream));
    }
    const uint64_t t = lane->dl_seq + 1;
    cudaEvent_t& e = lane->dl_done[t % hevcgpu_ctx::EVENT_RING];
    if (!e) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(e, lane->cstream));
    lane->dl_seq = t;
    *ticket = t;
    return HEVCGPU_OK;
}

int hevcgpu_lane_wait(hevcgpu_lane_t* lane, uint64_t ticket) {
    if (!lane) return fail(HEVCGPU_EINVAL, "null lane");
    if (ticket == 0 || ticket > lane->dl_seq) return fail(HEVCGPU_EINVAL, "unknown download ticket %llu",
                                                          (unsigned long long)ticket);
    CUDA_TRY(cudaEventSynchronize(lane->dl_done[ticket % hevcgpu_ctx::EVENT_RING]));
    return hevcgpu_ctx::take_status_of(lane->flow);
}

int hevcgpu_stream_sync(hevcgpu_stream_t* st) {
    if (!st) return fail(HEVCGPU_EINVAL, "null stream");
    CUDA_TRY(cudaStreamSynchronize(st->ctx->stream));
    return st->ctx->take_status();
}

int hevcgpu_profile_enable(hevcgpu_ctx_t* ctx, int enable) {
    if (!ctx) return fail(HEVCGPU_EINVAL, "null context");
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->profiling = enable != 0;
    ctx->marks.clear();
    ctx->ev_used = 0;
    return HEVCGPU_OK;
}

int hevcgpu_profile_read(hevcgpu_ctx_t* ctx, double* ms, uint64_t* launches) {
    if (!ctx) return fail(HEVCGPU_EINVAL, "null context");
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < HEVCGPU_NUM_STAGES; k++) {
        if (ms) ms[k] = 0;
        if (launches) launches[k] = 0;
    }
    for (auto& m : ctx->marks) {
        float t = 0;
        CUDA_TRY(cudaEventElapsedTime(&t, m.a, m.b));
        if (ms) ms[m.stage] += t;
        if (launches) launches[m.stage] += m.launches;
    }
    ctx->marks.clear();
    ctx->ev_used = 0;
    return HEVCGPU_OK;
}

int hevcgpu_picture_decode(hevcgpu_stream_t* st, const hevc_picture_syntax_t* syn, int32_t dst_slot) {
    hevcgpu_job_t* j = nullptr;
    int rc = hevcgpu_job_prepare(st, syn, &j);
    if (rc) return rc;
    rc = hevcgpu_job_launch(j, dst_slot);
    if (rc == HEVCGPU_OK) {
        cudaError_t e = cudaStreamSynchronize(st->ctx->stream);
        rc = e != cudaSuccess ? fail(HEVCGPU_ECUDA, "picture decode: %s", cudaGetErrorString(e))
                              : st->ctx->take_status();
    }
    hevcgpu_job_free(j);
    return rc;
}

}  // extern "C"
