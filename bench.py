"""Benchmark of the hevc.js B200 reconstruction back end.

Workload (one step): one 60-picture GOP of 8 streams of 1920x1080 4:2:0 8-bit pictures —
per stream an I picture, then 59 P/B pictures, each predicted from the stream's two
previous pictures in its HBM DPB (a ring of 3 slots) — reconstructed from seeded
synthetic picture syntax (CU quadtree split 0.5 to 8x8; P/B: 10 % intra CUs, 20 % skip,
50 % bi-prediction, 10 % explicit WP, MVs +-256 qpel; QP 22..37; SAO per CTU): motion
compensation, dequant + inverse transform, intra wavefront, deblocking, SAO.  The 8
streams' pictures of one GOP position are merged into one batch (one launch per stage);
the 60 batches run in decode order, each after the one it references.  The plain form
(one launch per stage per picture) is timed beside it.  Output is bit-exact against the
reference (checked by the tests; before timing, the bench checks every picture of the GOP
chain of every stream against the oracle, chaining the oracle's own outputs as references).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value      frames/s over the whole job with the records already in HBM: K GOPs, batched
           form, timed on the device from before the first batch to after the last (max
           over ranks).  "plain" is one launch per stage per picture on the same GOPs.
samples_per_s and alg_bytes_per_step: value in samples/s (W x H x 1.5 per picture) and the
           algorithmic bytes of a GOP summed over the stages.
frame_ms   device time of each GOP position's batch (all its pictures complete with it),
           p50 and p99 over the timed batches; i_frame_ms / pb_frame_ms split it by kind.
e2e        frames/s through the C ABI from host memory, as a decoder pipeline: per group of 4
           GOP positions the 32 pictures' records, kept in page-locked host memory
           (hevcgpu_host_alloc, as a recorder writing there would), are copied host->device
           with the work lists the library's host workers derive from them
           (hevcgpu_jobs_prepare_async), by a host thread that runs up to 2 groups ahead of
           the launches; the four batches of a group are launched in order on the streams'
           lane and every reconstructed picture is copied device->host into pinned frame
           buffers (hevcgpu_lane_slots_download_async, waited for with hevcgpu_lane_wait
           before the buffers come round again and at the end).  The median of three timed
           runs is reported, the three beside it.
stages     per-stage device times over one GOP from CUDA events recorded around each stage
           on the library's stream, in a separate pass (the timed region carries no extra
           events); the roofline is that of the dominant stage.
pb16       the P/B steady state: 2 groups of 16 streams of P/B pictures whose batches
           alternate over two lanes (consecutive batches overlap on the device), with its
           batched and plain forms and its own end-to-end rate.
serving    64 live streams of mixed resolutions with Poisson segment arrivals (4 lanes,
           continuous batching): per-frame latency p50/p99.
dropin     the drop-in decoder (hevc_decoder_decode, CABAC included) on the reference's 1080p
           stream, beside the reference's own build of the same API; dropin_generated the
           same on generated 1080p random-access streams, without and with WPP, in a child
           process bounded by a timeout.
--impl reference runs privaloops/hevc.js's own reconstruction functions (oracle/_ref,
           compiled from the reference's sources) on all host cores for the same GOP mix.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_DEFAULT, H_DEFAULT = 1920, 1080
PICTURE_CFG = dict(p_intra=0.1, p_skip=0.2, p_merge=0.3)
METRIC = "bit-exact 1080p frames/s on 1 B200, batched/served vs plain GPU; p50/p99 frame ms"
SLOTS = 3   # DPB ring per stream: picture n writes slot n % 3 and references the two before


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="GOPs timed")
    ap.add_argument("--warmup", type=int, default=3, help="GOPs run before timing")
    ap.add_argument("--streams", type=int, default=8, help="streams per batch (GOP workload)")
    ap.add_argument("--gop", type=int, default=60, help="pictures per GOP (an I picture, then P/B)")
    ap.add_argument("--batch", type=int, default=16, help="streams per batch of the P/B steady state")
    ap.add_argument("--width", type=int, default=W_DEFAULT)
    ap.add_argument("--height", type=int, default=H_DEFAULT)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-only", action="store_true", help="short run for ncu captures (batched launches only)")
    ap.add_argument("--workload", default="gop", choices=["gop", "pb16"],
                    help="--profile-only: GOP batches, or the P/B steady state's batches of --batch pictures")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving (Poisson) measurement")
    ap.add_argument("--no-pb16", action="store_true", help="skip the P/B steady-state measurement")
    ap.add_argument("--serve-seconds", type=float, default=6.0)
    ap.add_argument("--dropin-generated", action="store_true",
                    help="only the drop-in on the generated 1080p stream (the bench's child process)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# --------------------------------------------------------------------------- replicas
# With N > 1 ranks (one process per GPU under torchrun) every rank reconstructs its own
# streams: the work shards by stream with no data-path collective.  These helpers are the
# host side of that: the per-rank content seed, the max over ranks of a time, and the
# whole-job rate.

def rank_seed0(rank):
    """First content seed of a rank's streams; ranks never share a stream."""
    return 1000 + 100000 * rank


def max_over_ranks(x, world, device):
    """Max of a per-rank float over all ranks (all_reduce MAX on device: a CUDA device
    under NCCL, the CPU under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, seconds):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / seconds


# --------------------------------------------------------------------------- workload

def make_streams(hb, n, w, h, seed0):
    """n P/B pictures' syntax and their two reference pictures (content seeds per stream)."""
    pics, refs = [], []
    for i in range(n):
        seed = seed0 + 97 * i
        pics.append(hb.Picture(hb.default_cfg(w, h, seed, poc=8, **PICTURE_CFG)))
        refs.append([hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)])
    return pics, refs


def ref_slots_of(n):
    """(list-0, list-1) DPB slots that picture n >= 1 of a stream references."""
    a, b = (n - 1) % SLOTS, (n - 2) % SLOTS
    return [a, b], [b, a]


def make_gop(hb, n_streams, w, h, seed0):
    """Per stream: (I picture, P/B pictures by DPB phase n % 3, contents of its 3 slots
    before picture 0).  Picture n >= 1 of a stream uses the P/B syntax of its phase, whose
    reference slots are the two pictures before it."""
    gop = []
    for i in range(n_streams):
        seed = seed0 + 97 * i
        ipic = hb.Picture(hb.default_cfg(w, h, seed, slice_type=2, poc=0))
        pb = []
        for ph in range(SLOTS):
            pic = hb.Picture(hb.default_cfg(w, h, seed + 11 + ph, poc=8, **PICTURE_CFG))
            l0, l1 = ref_slots_of(ph + SLOTS)
            prm = pic.syn.params
            for k in range(prm.num_ref[0]):
                prm.ref_slot[0][k] = l0[k]
            for k in range(prm.num_ref[1]):
                prm.ref_slot[1][k] = l1[k]
            pb.append(pic)
        gop.append((ipic, pb, [hb.content(w, h, seed + 1 + s) for s in range(SLOTS)]))
    return gop


def gop_picture(stream, n):
    ipic, pb, _ = stream
    return ipic if n == 0 else pb[n % SLOTS]


def gop_sequence(gop, frames):
    """(picture, reference planes) of every picture of one GOP in decode order, position
    by position: the CPU arms' work list (every picture reads the stream's initial slots,
    so the pictures are independent there; the work per picture is the same)."""
    return [(gop_picture(s, n), s[2]) for n in range(frames) for s in gop]


def verify_gop_chain(hb, check, gop, sts, frame_jobs, frames):
    """Every picture of every stream of a GOP, reconstructed batch by batch in decode order,
    against the oracle's chain (each oracle picture predicted from the oracle's own earlier
    outputs).  Returns the list of mismatches (empty when bit-exact)."""
    import hashlib
    from concurrent.futures import ThreadPoolExecutor

    def oracle_chain(i):
        dpb = list(gop[i][2])
        out = []
        for n in range(frames):
            dpb[n % SLOTS] = check.reconstruct_picture(gop_picture(gop[i], n), dpb)
            out.append(hashlib.md5(dpb[n % SLOTS].tobytes()).hexdigest())
        return out

    with ThreadPoolExecutor(max_workers=len(gop)) as ex:
        want = list(ex.map(oracle_chain, range(len(gop))))
    errs = []
    buf = None
    for n in range(frames):
        hb.batch_launch(frame_jobs(n), [n % SLOTS] * len(gop))
        for i, st in enumerate(sts):
            buf = st.download(n % SLOTS, buf)
            if hashlib.md5(buf.tobytes()).hexdigest() != want[i][n]:
                errs.append(f"stream {i} picture {n} differs from the oracle")
    return errs


def algorithmic_bytes(hb, pic):
    """Algorithmic HBM bytes per stage of one picture (reads + writes the stage must do)."""
    import numpy as np
    s = pic.syn
    W, H = s.params.width, s.params.height
    npu, ntu = s.num_pus, s.num_tus

    def records(ptr, n, dtype):   # an array of n records at ptr (none for n == 0: ptr may be NULL)
        if n == 0:
            return np.zeros(0, dtype)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), (n * dtype.itemsize,)).view(dtype)

    pu = records(s.pus, npu, np.dtype([("x", "<u2"), ("y", "<u2"), ("w", "u1"), ("h", "u1"), ("r", "i1", 2),
                                       ("mv", "<i2", 4), ("wp", "<i2"), ("pad", "<u2")]))
    pw, ph = pu["w"].astype(np.int64), pu["h"].astype(np.int64)
    lists = (pu["r"] >= 0).sum(axis=1)
    mc_read = int((lists * ((pw + 7) * (ph + 7) + 2 * (pw // 2 + 3) * (ph // 2 + 3))).sum())
    mc_write = int((pw * ph * 3 // 2).sum())
    tu = records(s.tus, ntu, np.dtype([("x", "<u2"), ("y", "<u2"), ("l", "u1"), ("c", "u1"), ("qp", "u1"),
                                       ("f", "u1"), ("m", "u1"), ("r", "u1", 3), ("off", "<u4")]))
    n2 = (1 << tu["l"].astype(np.int64)) ** 2
    coded = (tu["f"] & 2) != 0
    intra = (tu["f"] & 1) != 0
    res = int((n2[coded & ~intra] * 4).sum() + (n2[coded & intra] * 4).sum())
    intra_b = int((n2 * intra).sum() + (2 * n2 * (intra & coded)).sum())
    pic_bytes = W * H * 3 // 2
    grid = (W // 4) * (H // 4) * 4
    return {"mc": mc_read + mc_write, "residual": res, "intra": intra_b,
            "deblock": 2 * pic_bytes + 2 * grid + (W // 4) * (H // 4) * 12, "sao": 2 * pic_bytes + grid}


# --------------------------------------------------------------------------- clocks

class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every 5 ms during the timed
    region (the device is found by its PCI bus id, so CUDA_VISIBLE_DEVICES remapping
    does not matter).  Falls back to `nvidia-smi -lms 200` when NVML is unavailable."""

    PERIOD_S = 0.005
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, local):
        self.local = local
        self.samples = []          # (sm_mhz, max_mhz, reasons bitmask)
        self.stop = threading.Event()
        self.nvml = None
        self.proc = None
        self.source = None

    def _handle(self):
        import pynvml
        import torch
        p = torch.cuda.get_device_properties(self.local)
        pynvml.nvmlInit()
        bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _sample_nvml(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((float(sm), float(mx), int(rs)))

    def _loop(self):
        while not self.stop.wait(self.PERIOD_S):
            try:
                self._sample_nvml()
            except Exception:
                return

    def __enter__(self):
        try:
            self.nvml = self._handle()
            self._sample_nvml()
            self.source = "nvml 5 ms"
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            fields = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                      "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                      "clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.local}", f"--query-gpu={fields}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi 200 ms"
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read_smi(self):
        bits = [0x8, 0x40, 0x20, 0x4]
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            try:
                rs = sum(b for b, v in zip(bits, parts[2:6]) if v.lower().startswith("active"))
                self.samples.append((float(parts[0]), float(parts[1]), rs))
            except (ValueError, IndexError):
                continue

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml:
            try:
                self._sample_nvml()
            except Exception:
                pass
            self.t.join(timeout=1)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": self.source}
        reasons = sorted(n for n, b in self.REASONS.items() if any(s[2] & b for s in self.samples))
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": self.source}


# --------------------------------------------------------------------------- CPU arms

_CPU_POOLS = {}


def cpu_run(checker, seq, first, n_pictures, threads):
    """Reconstruct n_pictures of the work list seq (round robin from index first) on host
    threads of a pool that persists across calls (its threads start once)."""
    from concurrent.futures import ThreadPoolExecutor
    ex = _CPU_POOLS.get(threads)
    if ex is None:
        ex = _CPU_POOLS[threads] = ThreadPoolExecutor(max_workers=threads)
        list(ex.map(lambda i: None, range(4 * threads)))   # start the threads
    t0 = time.perf_counter()
    list(ex.map(lambda i: checker.reconstruct_picture(*seq[(first + i) % len(seq)]), range(n_pictures)))
    return time.perf_counter() - t0


def cpu_checker():
    import oracle
    if oracle.ref_available():
        return oracle.ref(), "reference"
    return oracle.port(), "port"


def gop_workload_name(W, H, G, F):
    return (f"{W}x{H} 4:2:0 8-bit GOP reconstruction: {G} streams x {F} pictures (an I picture, then P/B "
            f"pictures predicted from the two before), MC + residual + intra wavefront + deblocking + SAO, "
            f"the {G} streams' pictures of a GOP position in one batch, batches in decode order")


def run_reference(args, hb, rank, world):
    """privaloops/hevc.js's own functions on the host cores, on the GOP mix: each step
    reconstructs the next `batch` pictures of the GOP work list."""
    if rank != 0:
        return None
    W, H, G, F, B = args.width, args.height, args.streams, args.gop, args.batch
    seq = gop_sequence(make_gop(hb, G, W, H, rank_seed0(0)), F)
    checker, kind = cpu_checker()
    threads = os.cpu_count() or 1
    pos = 0
    for _ in range(args.warmup):
        cpu_run(checker, seq, pos, B, threads)
        pos += B
    times = []
    for _ in range(args.steps):
        times.append(cpu_run(checker, seq, pos, B, threads))
        pos += B
    total = sum(times)
    value = B * args.steps / total
    line = {"metric": METRIC, "value": round(value, 3), "unit": "frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * total / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32",
            "data": "synthetic (seeded picture syntax and sinusoid reference pictures)", "impl": "reference",
            "config": {"workload": gop_workload_name(W, H, G, F), "global_batch": G,
                       "parallelism": f"{threads} host threads, one picture per thread",
                       "step": f"{B} consecutive pictures of the GOP work list"},
            "cpu_baseline": {"value": round(value, 3), "unit": "frames/s", "cores": threads, "kind": kind,
                             "sample": f"{B} pictures of the GOP mix per step x {args.steps} steps"},
            "e2e": {"value": round(value, 3), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


# --------------------------------------------------------------------------- GPU arm

import ctypes as C  # noqa: E402


def pct(v, q):
    s = sorted(v)
    return s[min(len(s) - 1, int(q * len(s)))] if s else None


def run_ours(args, hb, rank, world, local):
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    ctx = hb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.cuda_stream, device=dev)
    W, H, G, F = args.width, args.height, args.streams, args.gop
    if args.profile_only and args.workload == "pb16":
        # one set-up launch of B P/B pictures, then --steps batched launches of them
        pics, refs = make_streams(hb, args.batch, W, H, rank_seed0(rank))
        sts, js = [], []
        for i in range(args.batch):
            st = ctx.open_stream(W, H, 3)
            st.upload(0, refs[i][0])
            st.upload(1, refs[i][1])
            sts.append(st)
            js.append(st.prepare(pics[i]))
        for _ in range(1 + max(1, args.steps)):
            hb.batch_launch(js, [2] * args.batch)
        ctx.sync()
        return None
    import oracle
    check = oracle.port()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def rank_max(x):
        return max_over_ranks(x, world, dev)

    # ---- the GOP workload: G streams, records of their I and P/B pictures resident in HBM
    gop = make_gop(hb, G, W, H, rank_seed0(rank))
    gop_streams = []
    for ipic, pb, init in gop:
        st = ctx.open_stream(W, H, SLOTS)
        for s in range(SLOTS):
            st.upload(s, init[s])
        gop_streams.append(st)
    jobs_i = [st.prepare(s[0]) for st, s in zip(gop_streams, gop)]
    jobs_pb = [[st.prepare(s[1][ph]) for st, s in zip(gop_streams, gop)] for ph in range(SLOTS)]

    def frame_jobs(n):
        return jobs_i if n == 0 else jobs_pb[n % SLOTS]

    def gop_batched(evs=None):
        for n in range(F):
            if evs is not None:
                evs[n][0].record(stream)
            hb.batch_launch(frame_jobs(n), [n % SLOTS] * G)
            if evs is not None:
                evs[n][1].record(stream)

    def gop_plain():
        for n in range(F):
            for j in frame_jobs(n):
                j.launch(n % SLOTS)

    if args.profile_only:
        for _ in range(max(1, args.steps)):
            gop_batched()
        ctx.sync()
        return None

    # every picture of the GOP chain of every stream against the oracle, each predicted from
    # the oracle's own earlier outputs
    errs = verify_gop_chain(hb, check, gop, gop_streams, frame_jobs, F)
    if errs:
        raise SystemExit("bench: " + errs[0])

    # batched GOPs, timed on the library's stream
    K = args.steps
    for _ in range(args.warmup):
        gop_batched()
    ctx.sync()
    barrier()
    torch.cuda.synchronize()
    evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(F)]
           for _ in range(K)]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ctx.launches
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for k in range(K):
            gop_batched(evs[k])
        ev1.record(stream)
        ev1.synchronize()
    launches = ctx.launches - l0
    torch.cuda.synchronize()
    barrier()
    gop_ms = rank_max(ev0.elapsed_time(ev1))
    frame_ms = [[a.elapsed_time(b) for (a, b) in evs[k]] for k in range(K)]
    all_ms = [x for row in frame_ms for x in row]
    i_ms = [row[0] for row in frame_ms]
    pb_ms = [x for row in frame_ms for x in row[1:]]
    value = job_rate(G * F * K, world, gop_ms / 1000.0)

    # plain form over the same GOPs
    plain_k = max(2, K // 4)
    gop_plain()
    ctx.sync()
    barrier()
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pl0 = ctx.launches
    p0.record(stream)
    for _ in range(plain_k):
        gop_plain()
    p1.record(stream)
    p1.synchronize()
    plain_launches = ctx.launches - pl0
    barrier()
    plain_ms = rank_max(p0.elapsed_time(p1))
    plain_value = job_rate(G * F * plain_k, world, plain_ms / 1000.0)

    # stage profile over one GOP (separate pass; events between stages)
    ctx.profile(True)
    gop_batched()
    stages = ctx.profile_read()
    ctx.profile(False)

    # roofline of the dominant stage over the GOP
    import json as _json
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(_json.load(open(peaks_path))["hbm_gbs"]), "measured"
    alg_of = {}
    alg_sum = None
    for n in range(F):
        for s in gop:
            pic = gop_picture(s, n)
            if id(pic) not in alg_of:
                alg_of[id(pic)] = algorithmic_bytes(hb, pic)
            a = alg_of[id(pic)]
            alg_sum = dict(a) if alg_sum is None else {k: alg_sum[k] + a[k] for k in a}
    stage_ms = {"mc": stages["mc"][0], "residual": stages["residual"][0], "intra": stages["intra"][0],
                "deblock": stages["deblock_v"][0] + stages["deblock_h"][0], "sao": stages["sao"][0]}
    per_stage = {}
    for k, ms in stage_ms.items():
        gbs = alg_sum[k] / (ms / 1000.0) / 1e9 if ms > 0 else 0.0
        per_stage[k] = {"ms_per_gop": round(ms, 4), "alg_bytes_per_gop": alg_sum[k], "GB/s": round(gbs, 1),
                        "frac_of_hbm": round(gbs / peak, 4)}
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    # DRAM bytes (read + write) per batch of each stage's kernels on this workload, from one
    # ncu capture of a GOP of 2 streams at 1080p (ncu --metrics dram__bytes_read.sum,
    # dram__bytes_write.sum --clock-control none python bench.py --profile-only --steps 1
    # --warmup 0 --streams 2), scaled by 4 to 8 pictures per launch (each picture is
    # independent work), the GOP's total divided by its 60 batches; taken again whenever the
    # stage's kernels change
    ncu_dram_gop8 = {"mc": 57564587, "residual": 83248384, "intra": 26987537, "deblock": 78734404, "sao": 25038421}
    traffic = (ncu_dram_gop8[dom] if dom in ncu_dram_gop8 and (W, H, G, F) == (W_DEFAULT, H_DEFAULT, 8, 60)
               else None)

    # end to end through the C ABI from host memory, as a decoder pipeline: a host thread
    # prepares the records of groups of E2E_POS GOP positions (the pictures of every
    # stream) on the library's host workers, up to E2E_AHEAD groups ahead, while this
    # thread launches each group's batches in decode order on the streams' lane and queues
    # its frame copies into pinned host buffers; a group's buffers and jobs come round
    # again (and are freed) once its copies have landed
    import concurrent.futures
    E2E_POS, E2E_AHEAD, E2E_BUFS = 4, 2, 3
    lane = hb.Lane(ctx)
    frame_bytes = hb.i420_size(W, H)
    out_host = [[[torch.empty(frame_bytes, dtype=torch.uint8).pin_memory().numpy() for _ in range(G)]
                 for _ in range(E2E_POS)] for _ in range(E2E_BUFS)]
    for s in gop:   # records in page-locked memory (set up outside the timing)
        for pic in [s[0]] + s[1]:
            pic.pin()
    preparer = concurrent.futures.ThreadPoolExecutor(1)

    def e2e_prepare(n0):
        ns = [n for n in range(n0, n0 + E2E_POS) if n < F]
        pics = [gop_picture(s, n) for n in ns for s in gop]
        return ns, hb.prepare_batch(gop_streams * len(ns), pics, wait_uploads=False)

    def e2e_run(gops):
        """gops GOPs end to end; returns the host->device bytes per GOP."""
        groups = [n0 for _ in range(gops) for n0 in range(0, F, E2E_POS)]
        ahead = [preparer.submit(e2e_prepare, groups[q]) for q in range(min(E2E_AHEAD, len(groups)))]
        tickets, held = [None] * E2E_BUFS, [[] for _ in range(E2E_BUFS)]
        h2d = 0
        for q in range(len(groups)):
            ns, js = ahead[q].result()
            if q + E2E_AHEAD < len(groups):
                ahead.append(preparer.submit(e2e_prepare, groups[q + E2E_AHEAD]))
            h2d += sum(j.upload_bytes for j in js)
            b = q % E2E_BUFS
            if tickets[b] is not None:
                for t in tickets[b]:
                    lane.wait(t)
            for j in held[b]:
                j.free()
            tickets[b] = []
            for i, n in enumerate(ns):
                lane.batch_launch(js[i * G:(i + 1) * G], [n % SLOTS] * G)
                tickets[b].append(lane.download_batch_async(gop_streams, [n % SLOTS] * G, out_host[b][i]))
            held[b] = js
        for b in range(E2E_BUFS):
            if tickets[b] is not None:
                for t in tickets[b]:
                    lane.wait(t)
            for j in held[b]:
                j.free()
        return h2d // gops

    # the median of three timed runs of e2e_k GOPs: the host side shares its cores and
    # memory bandwidth with whatever else runs on the machine
    e2e_k = max(4, K // 2)
    e2e_run(1)
    e2e_times = []
    for _ in range(3):
        barrier()
        t0 = time.perf_counter()
        e2e_h2d = e2e_run(e2e_k)
        e2e_times.append(rank_max(time.perf_counter() - t0))
    e2e_s = statistics.median(e2e_times)
    preparer.shutdown()
    e2e_value = job_rate(G * F * e2e_k, world, e2e_s)

    clk = clocks.summary()
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "frames/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(gop_ms / K, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32", "data": "synthetic (seeded picture "
        "syntax and sinusoid reference pictures; no public dataset)",
        "config": {"workload": gop_workload_name(W, H, G, F), "global_batch": G * world,
                   "step": f"one GOP: {F} batches of {G} pictures", "parallelism":
                   f"replicas x{world} (streams sharded, no collective)",
                   "l2": "inputs larger than L2: a GOP's working set (the streams' DPB slots and the records "
                         "and work buffers of 4 x G prepared pictures) is several hundred MB; each batch reads "
                         "the pictures the batch before it wrote, as decoding does"},
        "plain": {"value": round(plain_value, 2), "unit": "frames/s",
                  "ms_per_picture": round(plain_ms / plain_k / (G * F), 4),
                  "gpu_launches_per_picture": round(plain_launches / plain_k / (G * F), 1)},
        "samples_per_s": round(value * W * H * 3 // 2),
        "alg_bytes_per_step": int(sum(alg_sum.values())),
        "batched_over_plain": round(value / plain_value, 3),
        "frame_ms": {"p50": round(statistics.median(all_ms), 4), "p99": round(pct(all_ms, 0.99), 4),
                     "note": "device time of a GOP position's batch; every picture of a batch completes with it"},
        "i_frame_ms": {"p50": round(statistics.median(i_ms), 4), "max": round(max(i_ms), 4)},
        "pb_frame_ms": {"p50": round(statistics.median(pb_ms), 4), "p99": round(pct(pb_ms, 0.99), 4)},
        "e2e": {"value": round(e2e_value, 2), "unit": "frames/s", "h2d_bytes_per_step": int(e2e_h2d),
                "d2h_bytes_per_step": int(G * F * frame_bytes),
                "runs": [round(job_rate(G * F * e2e_k, world, t), 1) for t in e2e_times],
                "note": "median of the three timed runs; the host preparation runs up to 2 groups of "
                        "4 GOP positions ahead of the launches, on its own thread"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": per_stage[dom]["GB/s"], "peak": peak,
                     "unit": "GB/s", "frac": per_stage[dom]["frac_of_hbm"],
                     "traffic": None if traffic is None else int(traffic),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, one capture",
                     "peak_source": peak_src},
        "stages": per_stage,
        "clocks": clk,
    }
    lane.close()
    if not args.no_pb16:
        line["pb16"] = run_pb16(args, hb, ctx, stream, rank, world, dev, check, rank_max, barrier)
    if not args.no_serving and rank == 0 and W == W_DEFAULT and H == H_DEFAULT:
        line["serving"] = run_serving(args, hb, local)
    if rank == 0 and not args.no_cpu_baseline:
        # last, so that its all-core host load is over before anything host-bound is timed
        checker, kind = cpu_checker()
        threads = os.cpu_count() or 1
        seq = gop_sequence(gop, F)
        # bounded sample: about 10 s of host work, whole GOPs of the same mix
        t_probe = cpu_run(checker, seq, 0, len(seq), threads)
        reps = max(1, int(round(10.0 / max(t_probe, 1e-3))))
        t = cpu_run(checker, seq, 0, reps * len(seq), threads)
        # one thread: a bounded sample (about 5 s) of pictures spread evenly over the GOP work
        # list, so that it holds I and P/B pictures in the GOP's proportion
        n1 = min(len(seq), max(G, int(round(5.0 / max(t_probe * threads / len(seq), 1e-4)))))
        t0_1 = time.perf_counter()
        for i in range(n1):
            checker.reconstruct_picture(*seq[(i * len(seq)) // n1])
        t1 = time.perf_counter() - t0_1
        line["cpu_baseline"] = {"value": round(reps * len(seq) / t, 3), "unit": "frames/s", "cores": threads,
                                "kind": kind, "sample": f"{reps} GOP(s) of {G} streams x {F} pictures "
                                f"({reps * len(seq)} pictures) on {threads} host threads ({t:.1f} s)",
                                "single_thread": {"value": round(n1 / t1, 3), "unit": "frames/s", "cores": 1,
                                                  "sample": f"{n1} pictures spread over the GOP work list on "
                                                            f"one thread ({t1:.1f} s)"}}
        line["dropin"] = run_dropin()
        line["dropin_generated"] = run_dropin_generated()
    for st in gop_streams:
        st.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return line if rank == 0 else None


DROPIN_STREAM = "bbb1080_50f.265"


def time_dropin(data, n, want_md5, reps=3):
    """Frames/s of hevc_decoder_decode (src/wasm/hevc_api.h:53) on one stream: the GPU drop-in
    (libhevcdec_gpu.so: NAL parsing, parameter sets, DPB logic and CABAC on this host thread,
    reconstruction on the GPU) beside the reference's own build of the same API
    (oracle/_ref/libhevcdec.so: its parser and its CPU reconstruction) on the same host; both
    outputs checked against want_md5, the MD5 of the stream's last n output frames.  The GPU
    decoder's context is made by an unmeasured decode of a 64x64 stream first (as a
    long-running process has it)."""
    import hashlib
    from hevc_b200 import decoder as D
    import oracle
    with open(os.path.join(ROOT, "tests", "golden", "streams", "toy_qp30.265"), "rb") as f:
        toy = f.read()

    def md5_of(frames):
        return hashlib.md5(b"".join(fr.yuv_bytes() for fr in frames[-n:])).hexdigest()

    out = {}
    ref_lib = os.path.join(oracle.HERE, "_ref", "libhevcdec.so")
    for name, lib, warm in (("gpu", None, True), ("reference", ref_lib, False)):
        if lib is not None and not os.path.exists(lib):
            out[name] = {"unavailable": f"{lib} is not built"}
            continue
        times, host, ok = [], [], True
        for _ in range(reps):
            dec = D.Decoder(lib)
            if warm and dec.decode(toy) != 0:
                raise SystemExit("bench: drop-in warm-up decode failed: " + dec.last_error())
            w0 = dec.gpu_wait_ns() if warm else 0
            t0 = time.perf_counter()
            rc = dec.decode(data)
            times.append(time.perf_counter() - t0)
            if warm:   # the decode call's own host time: its waits for the GPU back end taken out
                host.append(times[-1] - (dec.gpu_wait_ns() - w0) / 1e9)
            if rc != 0:
                raise SystemExit(f"bench: {name} decode failed: {dec.last_error()}")
            ok = ok and md5_of(dec.frames()) == want_md5
            dec.close()
        t = statistics.median(times)
        out[name] = {"frames_per_s": round(n / t, 2), "ms_per_frame": round(1000 * t / n, 3), "md5_ok": ok}
        if host:
            h = statistics.median(host)
            cores = os.cpu_count() or 1
            out[name]["host_ms_per_frame"] = round(1000 * h / n, 3)
            out[name]["host_frames_per_s_per_core"] = round(n / h, 2)
            out[name]["host_note"] = (
                "the decode call's time outside its waits for the GPU (hevc_decoder_gpu_wait_ns): NAL and "
                f"slice parsing, CABAC and the recording of each picture, on one core; {cores} such "
                f"decoders would parse about {round(cores * n / h)} pictures/s of this stream")
    if "frames_per_s" in out.get("reference", {}):
        out["gpu_over_reference"] = round(out["gpu"]["frames_per_s"] / out["reference"]["frames_per_s"], 2)
    return out


def run_dropin(reps=3):
    """The drop-in decoder on the reference's own 1080p stream (Big Buck Bunny, 50 pictures,
    I/P/B, scaling lists, SAO), checked against the reference's whole-stream MD5."""
    here = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(here, "streams.json")) as f:
        want = json.load(f)[DROPIN_STREAM]
    with open(os.path.join(here, "streams", DROPIN_STREAM), "rb") as f:
        data = f.read()
    n = len(want["frames"])
    out = {"stream": DROPIN_STREAM, "frames": n, "width": want["width"], "height": want["height"]}
    out.update(time_dropin(data, n, want["md5"], reps))
    out["note"] = ("the whole decode call, CABAC included: one host thread parses in both (the stream has no "
                   "WPP entry points), the GPU decoder reconstructs each picture while the next is parsed")
    return out


# The generated 1080p stream of the drop-in's second measurement: random-access mini-GOPs of
# 8 (reordered B pictures), cu_qp_delta, deblocking control, SAO, TMVP, AMP; levels and skip
# rates that give about 60 KB per picture.
GENERATED_1080P = dict(width=1920, height=1080, seed=4242, inter=1, pictures=32, ra_gop=8, p_b=0.8, max_refs=3,
                       log2_ctb=6, p_cbf=0.3, p_sig=0.15, max_level=40, qp_min=22, qp_max=37, qp_delta_depth=2,
                       deblock_ctl=1, p_skip=0.35, p_merge=0.5, p_intra_cu=0.05)


def dropin_generated_child(reps=3):
    """The drop-in on streams of the random-syntax generator (csrc/bitgen.cpp), in this
    process: GENERATED_1080P, and the same syntax with WPP (entry points per CTU row, which
    the reference's parser decodes on its thread pool, so both decoders parse on several
    host threads) under "wpp"."""
    out = generated_leg(GENERATED_1080P, reps)
    out["wpp"] = generated_leg(GENERATED_1080P_WPP, reps)
    out["wpp"]["note"] = ("the same syntax with WPP: one slice per picture, CTU rows parsed on the reference "
                          "parser's thread pool in both decoders")
    return out


# the WPP form of GENERATED_1080P (another seed)
GENERATED_1080P_WPP = dict(GENERATED_1080P, seed=4243, wpp=1)


def generated_leg(cfg, reps):
    """One generated stream through time_dropin: the reference's own decode gives the MD5
    both decoders are checked against."""
    import hashlib
    from hevc_b200 import bitgen, decoder as D
    import oracle
    c = dict(cfg)
    w, h, seed = c.pop("width"), c.pop("height"), c.pop("seed")
    data, pics = bitgen.generate(w, h, seed, **c)
    ref = D.Decoder(os.path.join(oracle.HERE, "_ref", "libhevcdec.so"))
    if ref.decode(data) != 0:
        raise SystemExit("bench: the reference cannot decode the generated stream: " + ref.last_error())
    frames = ref.frames()
    want = hashlib.md5(b"".join(fr.yuv_bytes() for fr in frames)).hexdigest()
    ref.close()
    out = {"stream": "generated (csrc/bitgen.cpp)", "config": cfg, "frames": len(frames),
           "bytes": len(data), "width": w, "height": h}
    out.update(time_dropin(data, len(frames), want, reps))
    out["note"] = ("random-access mini-GOPs of 8 from the seeded generator; both decoders checked against the "
                   "reference's own decode of the stream; the CABAC parse is the reference's on one host thread")
    return out


def run_dropin_generated(timeout_s=600):
    """dropin_generated_child in a child process (bench.py --dropin-generated), bounded by a
    timeout, so that this measurement cannot hold up or end the bench line."""
    import subprocess
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--dropin-generated"], capture_output=True,
                           text=True, timeout=timeout_s, cwd=ROOT)
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout_s} s"}
    lines = [ln for ln in r.stdout.strip().split("\n") if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": f"exit {r.returncode}: {(r.stderr or r.stdout)[-400:]}"}
    return json.loads(lines[-1])


def run_pb16(args, hb, ctx, stream, rank, world, dev, check, rank_max, barrier):
    """The P/B steady state: two groups of B streams with one prepared P/B picture each;
    their batches alternate over two lanes, so consecutive batches overlap on the device."""
    import numpy as np
    import torch
    W, H, B, K = args.width, args.height, args.batch, max(20, 5 * args.steps)
    slots = [2] * B

    def build_group(seed0):
        g_pics, g_refs = make_streams(hb, B, W, H, seed0)
        g_streams, g_jobs = [], []
        for i in range(B):
            st = ctx.open_stream(W, H, 3)
            st.upload(0, g_refs[i][0])
            st.upload(1, g_refs[i][1])
            g_streams.append(st)
            g_jobs.append(st.prepare(g_pics[i]))
        hb.batch_launch(g_jobs, slots)
        ctx.sync()
        for i in range(B):
            got = g_streams[i].download(2)
            want = check.reconstruct_picture(g_pics[i], g_refs[i])
            if not np.array_equal(got, want):
                raise SystemExit(f"bench: P/B picture {i} differs from the oracle in {int((got != want).sum())} samples")
        return g_pics, g_streams, g_jobs

    seed0 = rank_seed0(rank) + 70000
    pics_a, streams_a, jobs_a = build_group(seed0)
    pics_b, streams_b, jobs_b = build_group(seed0 + 50000)
    groups, grp_pics, grp_streams = [jobs_a, jobs_b], [pics_a, pics_b], [streams_a, streams_b]
    lanes = [hb.Lane(ctx), hb.Lane(ctx)]
    lane_st = [torch.cuda.ExternalStream(ln.cuda_stream, device=dev) for ln in lanes]

    for k in range(args.warmup):
        lanes[k % 2].batch_launch(groups[k % 2], slots)
    for ln in lanes:
        ln.sync()
    ctx.sync()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev0.record(lane_st[0])
    lane_st[1].wait_event(ev0)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    for k in range(K):
        i = k % 2
        starts[k].record(lane_st[i])
        lanes[i].batch_launch(groups[i], slots)
        ends[k].record(lane_st[i])
    for ln in lanes:
        ln.sync()
    torch.cuda.synchronize()
    barrier()
    served_ms = rank_max(max(ev0.elapsed_time(ends[K - 1]), ev0.elapsed_time(ends[K - 2])))
    batch_ms = [starts[k].elapsed_time(ends[k]) for k in range(K)]

    def timed(fn, steps):
        fn()
        ctx.sync()
        barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            fn()
        b.record(stream)
        b.synchronize()
        barrier()
        return rank_max(a.elapsed_time(b))

    batched_k, plain_k = max(3, K // 2), max(3, K // 4)
    batched_ms = timed(lambda: hb.batch_launch(jobs_a, slots), batched_k)
    plain_ms = timed(lambda: [j.launch(2) for j in jobs_a], plain_k)

    frame_bytes = hb.i420_size(W, H)
    out_host = [[torch.empty(frame_bytes, dtype=torch.uint8).pin_memory().numpy() for _ in range(B)]
                for _ in range(2)]
    for g_pics in grp_pics:
        for p in g_pics:
            p.pin()

    # end to end as a decoder pipeline, like the GOP workload's: a host thread prepares
    # the batches up to two ahead of the launches
    import concurrent.futures
    preparer = concurrent.futures.ThreadPoolExecutor(1)

    def e2e_prepare(i):
        return hb.prepare_batch(grp_streams[i], grp_pics[i], wait_uploads=False)

    def e2e_run(steps):
        ahead = [preparer.submit(e2e_prepare, k % 2) for k in range(min(2, steps))]
        tickets, held = [None, None], [[], []]
        for k in range(steps):
            i = k % 2
            js = ahead[k].result()
            if k + 2 < steps:
                ahead.append(preparer.submit(e2e_prepare, (k + 2) % 2))
            if tickets[i] is not None:
                lanes[i].wait(tickets[i])
                for j in held[i]:
                    j.free()
            lanes[i].batch_launch(js, slots)
            tickets[i] = lanes[i].download_batch_async(grp_streams[i], slots, out_host[i])
            held[i] = js
        for i in range(2):
            if tickets[i] is not None:
                lanes[i].wait(tickets[i])
                for j in held[i]:
                    j.free()

    e2e_k = max(16, K // 2)
    e2e_run(4)
    e2e_times = []
    for _ in range(3):
        barrier()
        t0 = time.perf_counter()
        e2e_run(e2e_k)
        e2e_times.append(rank_max(time.perf_counter() - t0))
    e2e_s = statistics.median(e2e_times)
    preparer.shutdown()
    for ln in lanes:
        ln.close()
    for st in streams_a + streams_b:
        st.close()
    return {"workload": f"{W}x{H} P/B pictures, 2 groups of {B} streams whose batches alternate over 2 lanes "
                        "(consecutive batches overlap on the device)",
            "value": round(job_rate(B * K, world, served_ms / 1000.0), 2), "unit": "frames/s", "steps": K,
            "batched": round(job_rate(B * batched_k, world, batched_ms / 1000.0), 2),
            "plain": round(job_rate(B * plain_k, world, plain_ms / 1000.0), 2),
            "frame_ms": {"p50": round(statistics.median(batch_ms), 4), "p99": round(pct(batch_ms, 0.99), 4)},
            "e2e": round(job_rate(B * e2e_k, world, e2e_s), 2)}


def run_serving(args, hb, local):
    """Live streams with Poisson segment arrivals (serve.run_poisson), latency ending when
    each frame has landed in page-locked host memory: the mixed-resolution load of the
    serving config, and 64 concurrent 1080p streams (the north-star latency target)."""
    from hevc_b200 import serve
    sctx = hb.Context(local)   # a serving process owns its context
    mixed = [(416, 240), (1280, 720), (1920, 1080), (3840, 2160)]
    pool = serve.PicturePool(hb, mixed, pin=True)
    out = {}
    for name, res, ratio in (("mixed", mixed, (4, 3, 2, 1)), ("1080p", [(1920, 1080)], (1,))):
        # an unmeasured 2 s run first: the first use of a context's pools and launch paths in
        # a process costs once what a long-running server pays at start-up
        serve.run_poisson(hb, sctx, seconds=2.0, n_streams=64, seed=5, lanes=4, pool=pool, resolutions=res,
                          ratio=ratio, download=True)
        r = serve.run_poisson(hb, sctx, seconds=args.serve_seconds, n_streams=64, seed=4, lanes=4, pool=pool,
                              resolutions=res, ratio=ratio, download=True)
        out[name] = {
            "streams": r["streams"], "hbm_bytes": r["hbm_bytes"], "frames": r["frames"],
            "frames_per_s": round(r["frames_per_s"], 1), "p50_ms": round(r["p50_ms"], 2),
            "p99_ms": round(r["p99_ms"], 2), "max_ms": round(r["max_ms"], 2),
            "steady_p50_ms": round(r["steady_p50_ms"], 2), "steady_p99_ms": round(r["steady_p99_ms"], 2),
            "frames_over_100ms": r["frames_over_100ms"], "worst_release_s": round(r["worst_release_s"], 3)}
    sctx.close()
    out["workload"] = ("64 live streams (mixed: 416x240 / 1280x720 / 1920x1080 / 3840x2160 in ratio 4:3:2:1; "
                       "1080p: all 1920x1080), 30 or 60 fps, 2-second segments (I picture, then P/B) arriving "
                       f"as a Poisson process (seed 4) for {args.serve_seconds:g} s; 4 lanes, continuous batching")
    out["latency"] = ("from the picture's live release time (segment start + i / fps) to the moment its frame "
                      "has landed in a page-locked host buffer (device event after the lane's copy); records "
                      "prepared on host workers, CABAC not included; frames/s is the offered load served; "
                      "measured after an unmeasured 2 s warm-up run on the same context")
    out["steady"] = ("frames released after the first 2 s, when every stream's first segment (and its I "
                     "picture) has arrived")
    return out


def main():
    args = parse()
    rank, world, local = dist_env()
    import __graft_entry__ as ge
    hb = ge.load_package()
    if args.dropin_generated:
        print(json.dumps(dropin_generated_child()), flush=True)
        return
    if args.impl == "reference":
        line = run_reference(args, hb, rank, world)
    else:
        line = run_ours(args, hb, rank, world, local)
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
