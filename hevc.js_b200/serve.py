"""Serving: continuous batching of many concurrent decode streams on one GPU context.

The request loop of a decoding service built on the C-ABI.  Streams of different
resolutions are admitted while their DPB slots and work buffers fit the context's HBM
budget; each admitted stream's DPB stays resident and the stream is pinned to one lane
(hevcgpu_lane_*), whose CUDA stream keeps its pictures in order.  Segments of pictures
arrive over time; a picture is *released* at its live time (segment arrival + i / fps).
Whenever a lane has room, the loop takes every stream of that lane whose next picture is
released, prepares their records in one batched call on the host workers
(hevcgpu_jobs_prepare) and launches them as one batch: pictures of many streams and
resolutions share the kernels, and batches on different lanes overlap on the device.
A picture's latency is its batch's completion on the device (CUDA event) minus its
release time.

The reference decoder has no counterpart: it decodes one stream, picture after picture
(Decoder::decode_picture, src/decoding/decoder.cpp:52-304).

Pictures come from the seeded syntax generator (one I picture per segment, P/B pictures
after it, two reference pictures in a three-slot DPB ring); CABAC parsing is not part
of this path and is not timed.
"""
import collections
import heapq
import random

import numpy as np

SLOTS = 3   # DPB ring per stream: picture n writes slot n % 3 and references the two before


def ref_slots_of(n):
    """(list-0, list-1) DPB slots that picture n of a stream references (n >= 1)."""
    a, b = (n - 1) % SLOTS, (n - 2) % SLOTS
    return [a, b], [b, a]


class PicturePool:
    """Generated syntax per resolution: one I picture and `variants` P/B pictures, each
    P/B one in SLOTS copies whose reference slots match picture index n % SLOTS."""

    def __init__(self, hb, resolutions, variants=2, seed=4, p_cfg=None):
        self.hb = hb
        self.pool = {}
        p_cfg = p_cfg or dict(p_intra=0.1, p_skip=0.2, p_merge=0.3)
        for (w, h) in resolutions:
            intra = hb.Picture(hb.default_cfg(w, h, seed + w + h, slice_type=2))
            pb = []
            for v in range(variants):
                by_phase = []
                for phase in range(SLOTS):
                    pic = hb.Picture(hb.default_cfg(w, h, seed + 31 * v + w, poc=8, **p_cfg))
                    l0, l1 = ref_slots_of(phase + SLOTS)   # n with n % SLOTS == phase, n >= 2
                    prm = pic.syn.params
                    for i in range(prm.num_ref[0]):
                        prm.ref_slot[0][i] = l0[i]
                    for i in range(prm.num_ref[1]):
                        prm.ref_slot[1][i] = l1[i]
                    by_phase.append(pic)
                pb.append(by_phase)
            self.pool[(w, h)] = (intra, pb)

    def picture(self, w, h, i, n, variant):
        """Syntax of picture i of a segment (i = 0: the I picture) that is picture n of its
        stream: a P/B picture whose reference slots are the two before slot n % SLOTS."""
        intra, pb = self.pool[(w, h)]
        if i == 0:
            return intra
        return pb[(variant + n) % len(pb)][n % SLOTS]


class _Stream:
    __slots__ = ("sid", "w", "h", "fps", "st", "lane", "queue", "n", "variant", "inflight")

    def __init__(self, sid, w, h, fps, st, lane, variant):
        self.sid, self.w, self.h, self.fps, self.st, self.lane = sid, w, h, fps, st, lane
        self.queue = collections.deque()   # (n within segment, release time)
        self.n = 0                          # pictures launched so far
        self.variant = variant
        self.inflight = 0


class Server:
    """Continuous batching over `lanes` lanes of one context.

    admit() opens a stream when its DPB and work buffers fit the budget (else False:
    the caller retries after streams close); add_segment() queues a segment's pictures
    with their release times; poll(now) launches and retires batches and returns the
    latencies (seconds) of the pictures completed since the last call."""

    def __init__(self, hb, ctx, pool, lanes=2, max_batch=64, depth=2, budget_bytes=None, content_seed=7):
        import torch
        self.hb, self.ctx, self.pool = hb, ctx, pool
        self.torch = torch
        self.lanes = [hb.Lane(ctx) for _ in range(lanes)]
        self.lane_cuda = [torch.cuda.ExternalStream(ln.cuda_stream) for ln in self.lanes]
        self.max_batch, self.depth = max_batch, depth
        self.budget = budget_bytes
        if budget_bytes:
            ctx.set_budget(budget_bytes)
        self.content_seed = content_seed
        self.streams = {}
        self.by_lane = [[] for _ in range(lanes)]
        self.inflight = [collections.deque() for _ in range(lanes)]
        self.frames_done = 0
        # device clock -> host clock: a base event recorded when the loop starts
        self.base_ev = None
        self.base_host = None

    # ---- clock
    def start_clock(self, now):
        torch = self.torch
        torch.cuda.synchronize()
        self.ctx.sync()
        self.base_ev = torch.cuda.Event(enable_timing=True)
        self.base_ev.record(self.lane_cuda[0])
        self.base_ev.synchronize()
        self.base_host = now

    def _device_time(self, ev):
        return self.base_host + self.base_ev.elapsed_time(ev) / 1000.0

    # ---- admission
    def stream_bytes(self, w, h):
        """HBM a stream holds: its DPB slots plus one picture's work buffers (records,
        reconstruction buffer, scratch) while a picture is in flight."""
        frame = self.hb.i420_size(w, h)
        return SLOTS * frame + 4 * frame

    def admit(self, sid, w, h, fps, variant=0):
        if self.budget is not None and self.ctx.bytes_in_use() + self.stream_bytes(w, h) > self.budget:
            return False
        try:
            st = self.ctx.open_stream(w, h, SLOTS)
        except self.hb.HevcGpuError as e:
            if e.code == self.hb.abi.HEVCGPU_ENOMEM:
                return False
            raise
        seed = self.content_seed + 1000 * sid
        for slot in range(1, SLOTS):   # the pictures the first segment's P/B pictures reach
            st.upload(slot, self.hb.content(w, h, seed + slot))
        lane = min(range(len(self.lanes)), key=lambda k: len(self.by_lane[k]))
        s = _Stream(sid, w, h, fps, st, lane, variant)
        self.streams[sid] = s
        self.by_lane[lane].append(s)
        return True

    def close_stream(self, sid):
        s = self.streams.pop(sid)
        self.lanes[s.lane].sync()
        self.by_lane[s.lane].remove(s)
        s.st.close()

    def add_segment(self, sid, arrival, n_pictures):
        s = self.streams[sid]
        for i in range(n_pictures):
            s.queue.append((i, arrival + i / s.fps))

    def pending(self):
        return sum(len(s.queue) for s in self.streams.values()) + sum(len(q) for q in self.inflight)

    # ---- the loop body
    def poll(self, now):
        done = []
        for k, q in enumerate(self.inflight):
            while q and q[0][0].query():
                ev, jobs, streams, releases = q.popleft()
                t_done = self._device_time(ev)
                for s, rel in zip(streams, releases):
                    done.append(t_done - rel)
                    s.inflight -= 1
                for j in jobs:
                    j.free()
                self.frames_done += len(jobs)
        for k, lane in enumerate(self.lanes):
            if len(self.inflight[k]) >= self.depth:
                continue
            ready = [s for s in self.by_lane[k] if s.queue and s.queue[0][1] <= now]
            if not ready:
                continue
            ready.sort(key=lambda s: s.queue[0][1])   # oldest release first
            ready = ready[: self.max_batch]
            pics, sts, slots, releases = [], [], [], []
            for s in ready:   # picture n of a stream writes slot n % SLOTS
                i, rel = s.queue.popleft()
                pics.append(self.pool.picture(s.w, s.h, i, s.n, s.variant))
                sts.append(s.st)
                slots.append(s.n % SLOTS)
                releases.append(rel)
            jobs = self.hb.prepare_batch(sts, pics)
            lane.batch_launch(jobs, slots)
            ev = self.torch.cuda.Event(enable_timing=True)
            ev.record(self.lane_cuda[k])
            for s in ready:
                s.n += 1
                s.inflight += 1
            self.inflight[k].append((ev, jobs, ready, releases))
        return done

    def drain(self):
        for ln in self.lanes:
            ln.sync()

    def close(self):
        self.drain()
        for sid in list(self.streams):
            self.close_stream(sid)
        for ln in self.lanes:
            ln.close()


def run_poisson(hb, ctx, seconds=5.0, n_streams=64, seed=4, lanes=2, max_batch=64, pool=None,
                resolutions=((416, 240), (1280, 720), (1920, 1080), (3840, 2160)), ratio=(4, 3, 2, 1),
                segment_s=2.0, clock=None):
    """Serve n_streams for `seconds` of wall time: resolutions in `ratio`, 30 or 60 fps,
    2-second segments arriving as a Poisson process per stream (mean gap = segment length,
    so each stream offers real-time load).  Returns latencies and throughput."""
    import time
    clock = clock or time.perf_counter
    rng = random.Random(seed)
    if pool is None:
        pool = PicturePool(hb, resolutions)
    srv = Server(hb, ctx, pool, lanes=lanes, max_batch=max_batch)
    mix = [r for r, k in zip(resolutions, ratio) for _ in range(k)]
    specs = []
    for sid in range(n_streams):
        w, h = mix[sid % len(mix)]
        fps = rng.choice((30, 60))
        specs.append((sid, w, h, fps))
    t0 = clock()
    srv.start_clock(t0)
    arrivals = []   # (time, sid)
    for sid, w, h, fps in specs:
        if not srv.admit(sid, w, h, fps, variant=sid):
            continue
        heapq.heappush(arrivals, (t0 + rng.expovariate(1.0 / segment_s) * 0.5, sid))
    lat = []
    offered = 0
    t_end = t0 + seconds
    while True:
        now = clock()
        while arrivals and arrivals[0][0] <= now and arrivals[0][0] < t_end:
            t, sid = heapq.heappop(arrivals)
            s = srv.streams[sid]
            n = int(round(segment_s * s.fps))
            srv.add_segment(sid, t, n)
            offered += n
            heapq.heappush(arrivals, (t + rng.expovariate(1.0 / segment_s), sid))
        lat.extend(srv.poll(now))
        if now >= t_end and srv.pending() == 0:
            break
    t_stop = clock()
    srv.close()
    lat_ms = np.array(lat) * 1000.0
    return {"streams": len(specs), "frames": int(len(lat)), "offered_frames": offered,
            "frames_per_s": len(lat) / (t_stop - t0), "p50_ms": float(np.percentile(lat_ms, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat_ms, 99)) if len(lat) else None,
            "max_ms": float(lat_ms.max()) if len(lat) else None, "wall_s": t_stop - t0}
