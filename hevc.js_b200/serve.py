"""Serving: continuous batching of many concurrent decode streams on one GPU context.

The request loop of a decoding service built on the C-ABI.  Streams of different
resolutions are admitted while their DPB slots and work buffers fit the context's HBM
budget; each admitted stream's DPB stays resident and the stream is pinned to one lane
(hevcgpu_lane_*), whose CUDA stream keeps its pictures in order.  Segments of pictures
arrive over time; a picture is *released* at its live time (segment start + i / fps, a
segment starting at its arrival or when the stream's previous segment ends).
Whenever a lane has room, the loop takes every stream of that lane whose next picture is
released, prepares their records in one batched call on the host workers
(hevcgpu_jobs_prepare) and launches them as one batch: pictures of many streams and
resolutions share the kernels, and batches on different lanes overlap on the device.
A picture's latency is its batch's completion on the device (CUDA event) minus its
release time; with downloads on, it ends instead when the picture's frame has landed in
page-locked host memory (the lane's asynchronous copies, hevcgpu_lane_slots_download_async,
timed by an event on the lane's copy stream), which is when a client could have it.

The reference decoder has no counterpart: it decodes one stream, picture after picture
(Decoder::decode_picture, src/decoding/decoder.cpp:52-304).

Pictures come from the seeded syntax generator (one I picture per segment, P/B pictures
after it, two reference pictures in a three-slot DPB ring); CABAC parsing is not part
of this path and is not timed.
"""
import collections
import concurrent.futures
import gc
import heapq
import os
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

    def __init__(self, hb, resolutions, variants=2, seed=4, p_cfg=None, pin=False):
        """pin: keep the pictures' large record arrays in page-locked memory (uploaded
        without a staging copy)."""
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
            if pin:
                for pic in [intra] + [q for ph in pb for q in ph]:
                    pic.pin()
            self.pool[(w, h)] = (intra, pb)

    def picture(self, w, h, i, n, variant):
        """Syntax of picture i of a segment (i = 0: the I picture) that is picture n of its
        stream: a P/B picture whose reference slots are the two before slot n % SLOTS."""
        intra, pb = self.pool[(w, h)]
        if i == 0:
            return intra
        return pb[(variant + n) % len(pb)][n % SLOTS]


class _Stream:
    __slots__ = ("sid", "w", "h", "fps", "st", "lane", "queue", "n", "n_queued", "variant", "inflight", "release_end")

    def __init__(self, sid, w, h, fps, st, lane, variant):
        self.sid, self.w, self.h, self.fps, self.st, self.lane = sid, w, h, fps, st, lane
        self.queue = collections.deque()   # [index in segment, release time, index in stream, prepared job]
        self.n = 0                          # pictures launched so far
        self.n_queued = 0                   # pictures queued so far
        self.variant = variant
        self.inflight = 0
        self.release_end = 0.0              # end of the release schedule of the queued segments


class Server:
    """Continuous batching over `lanes` lanes of one context.

    admit() opens a stream when its DPB and work buffers fit the budget (else False:
    the caller retries after streams close); add_segment() queues a segment's pictures
    with their release times; poll(now) launches and retires batches and returns the
    latencies (seconds) of the pictures completed since the last call.

    A picture's records are prepared (hevcgpu_job_prepare, on a pool of host threads) as
    soon as its segment is queued, up to `lookahead` pictures ahead per stream: preparing
    needs only the syntax, not the previous pictures, so launching never waits for it
    unless the preparation is slower than the stream."""

    def __init__(self, hb, ctx, pool, lanes=2, max_batch=64, depth=2, budget_bytes=None, content_seed=7,
                 lookahead=4, prep_threads=None, min_batch=1, max_wait=0.0, download=False):
        import torch
        self.hb, self.ctx, self.pool = hb, ctx, pool
        self.lookahead = lookahead
        self.prep = concurrent.futures.ThreadPoolExecutor(max_workers=prep_threads or os.cpu_count() or 4)
        self.torch = torch
        self.lanes = [hb.Lane(ctx) for _ in range(lanes)]
        self.lane_cuda = [torch.cuda.ExternalStream(ln.cuda_stream) for ln in self.lanes]
        # downloads: every picture's frame is copied into a page-locked host buffer of its
        # stream (a ring of `depth` + 2 per stream, so that no copy still in flight is
        # overwritten) and its latency ends when the copy has landed
        self.download = download
        self.lane_copy = [torch.cuda.ExternalStream(ln.copy_stream) for ln in self.lanes] if download else None
        self.frames = {}
        self.max_batch, self.depth = max_batch, depth
        # a lane launches when min_batch pictures are ready or the oldest ready one has
        # waited max_wait seconds since its release
        self.min_batch, self.max_wait = min_batch, max_wait
        self.budget = budget_bytes
        if budget_bytes:
            ctx.set_budget(budget_bytes)
        self.content_seed = content_seed
        self.streams = {}
        self.by_lane = [[] for _ in range(lanes)]
        self.inflight = [collections.deque() for _ in range(lanes)]
        self.frames_done = 0
        self.batches = []   # (lane, pictures, launch time, completion time) of finished batches
        self.records = []   # (release time, latency, stream id) of finished pictures
        # device clock -> host clock: a base event recorded when the loop starts
        self.base_ev = None
        self.base_host = None

    # ---- clock
    def start_clock(self, clock):
        """Tie the device clock to the host clock `clock()`; returns the host time."""
        torch = self.torch
        torch.cuda.synchronize()
        self.ctx.sync()
        self.base_ev = torch.cuda.Event(enable_timing=True)
        self.base_ev.record(self.lane_cuda[0])
        self.base_ev.synchronize()
        self.base_host = clock()
        return self.base_host

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
        if self.download:
            size = self.hb.i420_size(w, h)
            self.frames[sid] = [self.torch.empty(size, dtype=self.torch.uint8).pin_memory().numpy()
                                for _ in range(self.depth + 2)]
        self.streams[sid] = s
        self.by_lane[lane].append(s)
        return True

    def close_stream(self, sid):
        s = self.streams.pop(sid)
        self.lanes[s.lane].sync()
        self.by_lane[s.lane].remove(s)
        s.st.close()

    def add_segment(self, sid, arrival, n_pictures):
        """Queue a segment.  A stream's segments follow each other in media time: frame i
        is released at start + i / fps, where start is the segment's arrival, or the end
        of the previous segment's frames if that is later (the segment arrived early and
        waits in the buffer)."""
        s = self.streams[sid]
        start = max(arrival, s.release_end)
        for i in range(n_pictures):
            s.queue.append([i, start + i / s.fps, s.n_queued, None])
            s.n_queued += 1
        s.release_end = start + n_pictures / s.fps
        self._feed(s)

    def _feed(self, s):
        """Start the preparation of the stream's next `lookahead` queued pictures."""
        for e in list(s.queue)[: self.lookahead]:
            if e[3] is None:
                pic = self.pool.picture(s.w, s.h, e[0], e[2], s.variant)
                e[3] = self.prep.submit(self.hb.Job, s.st, pic)

    def warm(self):
        """Fill the context's device and pinned pools before serving: prepare the first
        `lookahead` pictures of every stream (its I picture and P/B pictures) at once and
        free them, so that the buffers the steady state needs are already allocated."""
        futs = []
        for s in self.streams.values():
            for n in range(self.lookahead):
                futs.append(self.prep.submit(self.hb.Job, s.st, self.pool.picture(s.w, s.h, n, n, s.variant)))
        jobs = [f.result() for f in futs]
        for j in jobs:
            j.free()

    def pending(self):
        return sum(len(s.queue) for s in self.streams.values()) + sum(len(q) for q in self.inflight)

    # ---- the loop body
    def poll(self, now):
        done = []
        for k, q in enumerate(self.inflight):
            while q and q[0][0].query():
                ev, jobs, streams, releases, t_launch = q.popleft()
                t_done = self._device_time(ev)
                self.batches.append((k, len(jobs), t_launch, t_done))
                for s, rel in zip(streams, releases):
                    done.append(t_done - rel)
                    self.records.append((rel, t_done - rel, s.sid))
                    s.inflight -= 1
                for j in jobs:
                    j.free()
                self.frames_done += len(jobs)
        for k, lane in enumerate(self.lanes):
            if len(self.inflight[k]) >= self.depth:
                continue
            ready = [s for s in self.by_lane[k]
                     if s.queue and s.queue[0][1] <= now and s.queue[0][3] is not None and s.queue[0][3].done()]
            if not ready:
                continue
            ready.sort(key=lambda s: s.queue[0][1])   # oldest release first
            if len(ready) < self.min_batch and now - ready[0].queue[0][1] < self.max_wait:
                continue
            ready = ready[: self.max_batch]
            jobs, slots, releases = [], [], []
            for s in ready:   # picture n of a stream writes slot n % SLOTS
                i, rel, n, fut = s.queue.popleft()
                jobs.append(fut.result())
                slots.append(n % SLOTS)
                releases.append(rel)
                self._feed(s)
            lane.batch_launch(jobs, slots)
            ev = self.torch.cuda.Event(enable_timing=True)
            if self.download:
                outs = [self.frames[s.sid][s.n % len(self.frames[s.sid])] for s in ready]
                lane.download_batch_async([s.st for s in ready], slots, outs)
                ev.record(self.lane_copy[k])
            else:
                ev.record(self.lane_cuda[k])
            for s in ready:
                s.n += 1
                s.inflight += 1
            self.inflight[k].append((ev, jobs, ready, releases, now))
        return done

    def drain(self):
        for ln in self.lanes:
            ln.sync()

    def close(self):
        self.drain()
        self.prep.shutdown(wait=True)
        for s in self.streams.values():   # prepared, never launched
            for e in s.queue:
                if e[3] is not None:
                    e[3].result().free()
        for sid in list(self.streams):
            self.close_stream(sid)
        for ln in self.lanes:
            ln.close()


def run_poisson(hb, ctx, seconds=5.0, n_streams=64, seed=4, lanes=4, max_batch=64, pool=None,
                resolutions=((416, 240), (1280, 720), (1920, 1080), (3840, 2160)), ratio=(4, 3, 2, 1),
                segment_s=2.0, clock=None, min_batch=8, max_wait=0.004, download=False):
    """Serve n_streams whose segments arrive for `seconds` of wall time (the run ends when
    every queued frame is decoded): resolutions in `ratio`, 30 or 60 fps, 2-second
    segments arriving as a Poisson process per stream (mean gap = segment length, so each
    stream offers real-time load).  Returns per-frame latency percentiles (device
    completion minus release) and the frames/s served."""
    import time
    clock = clock or time.perf_counter
    rng = random.Random(seed)
    if pool is None:
        pool = PicturePool(hb, resolutions)
    srv = Server(hb, ctx, pool, lanes=lanes, max_batch=max_batch, min_batch=min_batch, max_wait=max_wait,
                 download=download)
    mix = [r for r, k in zip(resolutions, ratio) for _ in range(k)]
    specs = []
    for sid in range(n_streams):
        w, h = mix[sid % len(mix)]
        fps = rng.choice((30, 60))
        specs.append((sid, w, h, fps))
    admitted = [sid for sid, w, h, fps in specs if srv.admit(sid, w, h, fps, variant=sid)]
    srv.warm()
    hbm = ctx.bytes_in_use()
    # the loop allocates no cycles; a cyclic collection pass over the whole process's
    # objects would stall it (for a long-running process holding many objects, by
    # hundreds of ms), so collect once now and keep the collector off while serving
    gc.collect()
    gc_was_on = gc.isenabled()
    gc.disable()
    try:
        t0 = srv.start_clock(clock)   # streams are open and their DPBs resident before the clock starts
        arrivals = []   # (time, sid): each stream's first segment within the first segment length
        for sid in admitted:
            heapq.heappush(arrivals, (t0 + rng.uniform(0.0, segment_s), sid))
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
    finally:
        if gc_was_on:
            gc.enable()
    records = np.array([(r[0], r[1]) for r in srv.records]) if srv.records else np.zeros((0, 2))
    srv.close()
    lat_ms = np.array(lat) * 1000.0
    # steady state: frames released after every stream's first segment has started (the
    # first segments, each opening with an I picture, all arrive within segment_s)
    steady = records[records[:, 0] >= t0 + segment_s, 1] * 1000.0 if len(records) else np.zeros(0)
    pct = lambda v, q: float(np.percentile(v, q)) if len(v) else None
    return {"streams": len(admitted), "hbm_bytes": int(hbm), "frames": int(len(lat)), "offered_frames": offered,
            "frames_per_s": len(lat) / (t_stop - t0), "p50_ms": pct(lat_ms, 50), "p99_ms": pct(lat_ms, 99),
            "max_ms": float(lat_ms.max()) if len(lat) else None, "steady_frames": int(len(steady)),
            "frames_over_100ms": int((records[:, 1] > 0.1).sum()) if len(records) else 0,
            "worst_release_s": float(records[records[:, 1].argmax(), 0] - t0) if len(records) else 0.0,
            "steady_p50_ms": pct(steady, 50), "steady_p99_ms": pct(steady, 99), "wall_s": t_stop - t0}
