// intra.cuh — intra prediction as a dataflow over transform units.
//
// Every intra TU reads reference samples left of and above it (build_reference_samples,
// intra_prediction.cpp:44-211).  The host lists, for each intra TU, the earlier intra TUs
// that own any of those samples (the only samples that are not final when this kernel
// starts: MC and the inter residuals ran before).  That DAG replaces the CTU wavefront:
//
//   k_intra_arm   re-arms the dependency counters and seeds a device queue with the TUs
//                 that wait for nothing;
//   k_intra_flow  persistent warps claim queue slots in order, wait (bounded) until their
//                 slot is published, predict the TU (reference samples, substitution,
//                 smoothing, planar/DC/angular, + residual, clip) straight into the
//                 picture, then count down their dependents and publish those that became
//                 ready.
//
// Progress is guaranteed without co-residency: a warp only waits for slot t after slots
// 0..t-1 were claimed by warps that are already running, and once those TUs are done some
// remaining TU has all its dependencies met (the graph is acyclic), so slot t gets
// published.  Every wait is bounded anyway: after SPIN_LIMIT polls the warp sets
// ST_TIMEOUT (in the launch state, which stops the other warps, and in the context's
// sticky status word that the host turns into HEVCGPU_ETIMEOUT) and returns.
#pragma once

#include <cuda/atomic>

#include "device_common.cuh"

namespace hevcgpu {

__constant__ int8_t c_intra_angle[35] = {0,   0,   32,  26,  21,  17,  13,  9,  5,  2,  0,  -2,
                                         -5,  -9,  -13, -17, -21, -26, -32, -26, -21, -17, -13, -9,
                                         -5,  -2,  0,   2,   5,   9,   13,  17,  21,  26,  32};
__constant__ int16_t c_inv_angle[35] = {0,    0,    256, 315, 390, 482,  630,  910,  1638, 4096, 0,   4096,
                                        1638, 910,  630, 482, 390, 315,  256,  315,  390,  482,  630, 910,
                                        1638, 4096, 0,   4096, 1638, 910, 630, 482,  390,  315,  256};

struct IntraWarpSmem {
    int16_t raw[129];  // reference samples as read (0 where unavailable)
    int16_t s[129];    // after substitution: bottom-left .. corner (index 2n) .. top-right
    int16_t f[129];    // after smoothing
};

// Predict + reconstruct one intra TU with one warp (perform_intra_prediction,
// intra_prediction.cpp:428-481, then reconstruct_block's add and clip).  Reference
// samples are read through L2 (ld.global.cg): other warps of this launch wrote them.
__device__ void intra_tu(const PicDesc& P, const hevc_tu_t& t, int lane, IntraWarpSmem& W) {
    const int ci = t.c_idx, sub = ci ? 2 : 1;
    const int n = 1 << t.log2_size, log2 = t.log2_size;
    const int xc = t.x, yc = t.y;
    const int ctb = 1 << P.log2_ctb, ctbc = ctb / sub;
    const int rx = xc / ctbc, ry = yc / ctbc;
    const int cur_addr = ry * P.wctb + rx;
    const int pw = P.width / sub, ph = P.height / sub;
    const int ox = rx * ctb, oy = ry * ctb;
    const int pitch = ci ? P.pitch_c : P.pitch_y;
    uint8_t* plane = P.rec + (ci == 0 ? 0 : (ci == 1 ? P.off_cb : P.off_cr));
    const int cur_slice = P.ctb_slice ? P.ctb_slice[cur_addr] : 0;
    const int cur_tile = P.ctb_tile ? P.ctb_tile[cur_addr] : 0;
    const uint32_t cur_z = zorder16((uint32_t)((xc * sub - ox) >> 2), (uint32_t)((yc * sub - oy) >> 2));
    const int total = 4 * n + 1;

    // 1. reference samples and their availability: in the picture, and either in an
    //    earlier CTB of the same slice and tile, or in this CTB at a lower z-scan address
    //    of the 4x4 luma unit (intra_prediction.cpp:102-133)
    uint32_t mask[5];
#pragma unroll
    for (int r = 0; r < 5; r++) {
        const int i = lane + 32 * r;
        bool ok = false;
        int val = 0;
        if (i < total) {
            int px, py;
            if (i < 2 * n) { px = xc - 1; py = yc + 2 * n - 1 - i; }
            else if (i == 2 * n) { px = xc - 1; py = yc - 1; }
            else { px = xc + (i - 2 * n - 1); py = yc - 1; }
            if (px >= 0 && py >= 0 && px < pw && py < ph) {
                const int ncx = px / ctbc, ncy = py / ctbc;
                if (ncx != rx || ncy != ry) {
                    const int a = ncy * P.wctb + ncx;
                    ok = a < cur_addr && (P.ctb_slice ? P.ctb_slice[a] : 0) == cur_slice &&
                         (P.ctb_tile ? P.ctb_tile[a] : 0) == cur_tile;
                } else {
                    ok = zorder16((uint32_t)((px * sub - ox) >> 2), (uint32_t)((py * sub - oy) >> 2)) < cur_z;
                }
                if (ok) val = __ldcg(plane + (int64_t)py * pitch + px);
            }
            W.raw[i] = (int16_t)val;
        }
        mask[r] = __ballot_sync(0xffffffffu, ok);
    }
    __syncwarp();
    // 2. substitution (:177-197): an unavailable sample takes the nearest available one
    //    below it in the array, or the first available one; none available -> 128
    int first = -1;
#pragma unroll
    for (int r = 0; r < 5; r++)
        if (first < 0 && mask[r]) first = 32 * r + __ffs(mask[r]) - 1;
#pragma unroll
    for (int r = 0; r < 5; r++) {
        const int i = lane + 32 * r;
        if (i >= total) continue;
        int v;
        if (first < 0) v = 128;
        else if ((mask[r] >> lane) & 1u) v = W.raw[i];
        else {
            int j = -1;
            const uint32_t m = lane ? (mask[r] & ((1u << lane) - 1u)) : 0u;
            if (m) j = 32 * r + 31 - __clz(m);
            for (int q = r - 1; q >= 0 && j < 0; q--)
                if (mask[q]) j = 32 * q + 31 - __clz(mask[q]);
            v = W.raw[j < 0 ? first : j];
        }
        W.s[i] = (int16_t)v;
    }
    __syncwarp();
    // 3. smoothing of luma references (:217-257, :443-471): [1 2 1] over the linear array
    //    (which also gives the corner filter), or the bilinear strong smoothing of 32x32
    const int mode = t.intra_mode;
    const int16_t* R = W.s;
    if (ci == 0 && !P.intra_smoothing_disabled && mode != 1 && n != 4) {
        const int d = min(abs(mode - 26), abs(mode - 10));
        const int thr = n == 8 ? 7 : (n == 16 ? 1 : 0);
        if (d > thr) {
            bool bil = false;
            if (P.strong_intra && n == 32) {
                const int c = W.s[2 * n];
                bil = abs(c + W.s[4 * n] - 2 * W.s[3 * n]) < 8 && abs(c + W.s[0] - 2 * W.s[n]) < 8;
            }
#pragma unroll
            for (int r = 0; r < 5; r++) {
                const int i = lane + 32 * r;
                if (i >= total) continue;
                int v;
                if (i == 0 || i == 4 * n) v = W.s[i];
                else if (bil) {
                    if (i == 2 * n) v = W.s[i];
                    else if (i > 2 * n) { int k = i - 2 * n; v = ((2 * n - k) * W.s[2 * n] + k * W.s[4 * n] + n) >> (log2 + 1); }
                    else { int k = 2 * n - i; v = ((2 * n - k) * W.s[2 * n] + k * W.s[0] + n) >> (log2 + 1); }
                } else {
                    v = (W.s[i - 1] + 2 * W.s[i] + W.s[i + 1] + 2) >> 2;
                }
                W.f[i] = (int16_t)v;
            }
            __syncwarp();
            R = W.f;
        }
    }
    // 4. prediction (top[k] = R[2n + k], left[k] = R[2n - k]) + residual, clip, store
    const int16_t* res = (t.flags & HEVC_TU_CODED) ? P.resid + t.coeff_offset : nullptr;
    const int ang = c_intra_angle[mode];
    const int inv = c_inv_angle[mode];
    int dc = 0;
    if (mode == 1) {  // predict_dc :295-317
        int s = 0;
        for (int i = lane; i < n; i += 32) s += R[2 * n + 1 + i] + R[2 * n - 1 - i];
        s = __reduce_add_sync(0xffffffffu, s);
        dc = (s + n) >> (log2 + 1);
    }
    for (int e = lane; e < n * n; e += 32) {
        const int y = e >> log2, x = e & (n - 1);
        int p;
        if (mode == 0) {  // predict_planar :263-289
            p = ((n - 1 - x) * R[2 * n - 1 - y] + (x + 1) * R[3 * n + 1] + (n - 1 - y) * R[2 * n + 1 + x] +
                 (y + 1) * R[n - 1] + n) >> (log2 + 1);
        } else if (mode == 1) {
            p = dc;
            if (ci == 0 && n < 32) {
                if (x == 0 && y == 0) p = (R[2 * n + 1] + R[2 * n - 1] + 2 * dc + 2) >> 2;
                else if (y == 0) p = (R[2 * n + 1 + x] + 3 * dc + 2) >> 2;
                else if (x == 0) p = (R[2 * n - 1 - y] + 3 * dc + 2) >> 2;
            }
        } else {  // predict_angular :323-422
            const bool vert = mode >= 18;
            const int pos = vert ? y : x, ln = vert ? x : y;
            const int idx = ((pos + 1) * ang) >> 5, fr = ((pos + 1) * ang) & 31;
            const int ri = ln + 1 + idx;
            // main reference (top for vertical, left for horizontal); negative indices
            // project onto the side reference through invAngle (:346-368)
            auto ref_at = [&](int q) -> int {
                if (q >= 0) return vert ? R[2 * n + q] : R[2 * n - q];
                const int si = min(2 * n, ((-q) * inv + 128) >> 8);
                return vert ? R[2 * n - si] : R[2 * n + si];
            };
            p = fr ? ((32 - fr) * ref_at(ri) + fr * ref_at(ri + 1) + 16) >> 5 : ref_at(ri);
            if (ci == 0 && n < 32) {
                if (mode == 26 && x == 0) p = clip_u8(p + ((R[2 * n - 1 - y] - R[2 * n]) >> 1));
                else if (mode == 10 && y == 0) p = clip_u8(p + ((R[2 * n + 1 + x] - R[2 * n]) >> 1));
            }
        }
        plane[(int64_t)(yc + y) * pitch + xc + x] = (uint8_t)clip_u8(p + (res ? res[e] : 0));
    }
}

constexpr int IF_WARPS = 8;
constexpr long long SPIN_LIMIT = 1ll << 23;  // polls of ~128 ns: about a second

__device__ __forceinline__ int32_t encode_item(int seg, int idx) { return (seg << 24) | idx; }

// Re-arm the counters of every picture and seed the queue: picture k's ready TUs go to
// slots [aux0, aux0 + n_ready), its other slots [n_ready_total + aux1 - aux0, ...) are
// cleared to -1 (aux0 = ready TUs of earlier pictures, aux1 = intra TUs of earlier ones).
__global__ void k_intra_arm(const __grid_constant__ SegTable st, FlowState* fs, int32_t* queue, int n_ready_total) {
    const Seg& sg = st.s[blockIdx.y];
    const PicDesc& P = *sg.pic;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        fs->head = 0;
        fs->tail = n_ready_total;
        fs->status = 0;
    }
    if (i >= P.n_intra) return;
    P.count[i] = P.init_count[i];
    if (i < P.n_ready) queue[sg.aux0 + i] = encode_item(blockIdx.y, P.ready[i]);
    else queue[n_ready_total + sg.aux1 - sg.aux0 + (i - P.n_ready)] = -1;
}

__global__ void __launch_bounds__(32 * IF_WARPS) k_intra_flow(const __grid_constant__ SegTable st, FlowState* fs,
                                                              int32_t* queue, int total, uint32_t* sticky) {
    __shared__ IntraWarpSmem ws[IF_WARPS];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    IntraWarpSmem& W = ws[warp];
    cuda::atomic_ref<int32_t, cuda::thread_scope_device> head(fs->head), tail(fs->tail);
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> status(fs->status);
    while (true) {
        int slot = 0, item = -1;
        if (lane == 0) {
            slot = head.fetch_add(1, cuda::memory_order_relaxed);
            if (slot < total) {
                cuda::atomic_ref<int32_t, cuda::thread_scope_device> q(queue[slot]);
                long long polls = 0;
                while ((item = q.load(cuda::memory_order_acquire)) < 0) {
                    if (status.load(cuda::memory_order_relaxed) != 0u || ++polls > SPIN_LIMIT) {
                        status.fetch_or(ST_TIMEOUT, cuda::memory_order_relaxed);
                        atomicOr(sticky, ST_TIMEOUT);
                        item = -1;
                        break;
                    }
                    __nanosleep(128);
                }
            }
        }
        slot = __shfl_sync(0xffffffffu, slot, 0);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (slot >= total || item < 0) return;
        const int seg = item >> 24, idx = item & 0xFFFFFF;
        const PicDesc& P = *st.s[seg].pic;
        const hevc_tu_t t = P.tus[P.intra_list[idx]];
        intra_tu(P, t, lane, W);
        // make this TU's samples visible before its dependents can be claimed
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            for (int k = P.dep_off[idx]; k < P.dep_off[idx + 1]; k++) {
                const int d = P.dep_list[k];
                cuda::atomic_ref<int32_t, cuda::thread_scope_device> cnt(P.count[d]);
                if (cnt.fetch_sub(1, cuda::memory_order_acq_rel) == 1) {
                    const int s2 = tail.fetch_add(1, cuda::memory_order_relaxed);
                    cuda::atomic_ref<int32_t, cuda::thread_scope_device> q(queue[s2]);
                    q.store(encode_item(seg, d), cuda::memory_order_release);
                }
            }
        }
        __syncwarp();
    }
}

}  // namespace hevcgpu
