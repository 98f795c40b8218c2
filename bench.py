"""Benchmark of the hevc.js B200 reconstruction back end.

Workload (one step): reconstruct B 1920x1080 4:2:0 8-bit pictures — motion
compensation from two reference pictures held in the HBM DPB, dequant + inverse
transform, intra wavefront, deblocking, SAO — from seeded synthetic P/B picture syntax
(CU quadtree split 0.5 to 8x8, 10 % intra CUs, 20 % skip, 50 % bi-prediction, 10 %
explicit WP, MVs +-256 qpel, QP 22..37, SAO per CTU), one picture per stream, B streams
merged into shared launches (the batched form).  The plain form (one launch per stage
per picture) is timed beside it and reported as "plain".  Output is bit-exact against
the reference (checked by the tests; the bench verifies one picture per stream against
the oracle before timing).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]

value      frames/s over the whole job with the records already in HBM, served form: two
           groups of B streams whose batches alternate over two lanes (hevcgpu_lane_*), so
           consecutive batches overlap on the device (device time from an event both lanes
           wait for to the later lane's last event, max over ranks).  "batched" is the same
           batches on one queue; "plain" one launch per stage per picture.
e2e        frames/s through the C ABI from host memory: per step the pictures' records, kept
           in page-locked host memory (hevcgpu_host_alloc, as a recorder writing there would),
           are copied host->device with the work lists the library's host workers derive from
           them (hevcgpu_jobs_prepare), the batch is launched on a lane, and every reconstructed
           picture is copied device->host into pinned host frame buffers
           (hevcgpu_lane_slots_download_async, waited for with hevcgpu_lane_wait before the
           buffers are reused two steps later and at the end); consecutive steps alternate
           lanes, so step k's host preparation overlaps step k-1 on the device and its copies.
stages     per-stage device times from CUDA events recorded around each stage on the
           library's stream, in a separate pass of the same batched step (the timed region
           itself carries no extra events).
--impl reference runs privaloops/hevc.js's own reconstruction functions (oracle/_ref,
           compiled from the reference's sources) on all host cores for the same workload.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--width", type=int, default=W_DEFAULT)
    ap.add_argument("--height", type=int, default=H_DEFAULT)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-only", action="store_true", help="short run for ncu captures")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving (Poisson) measurement")
    ap.add_argument("--serve-seconds", type=float, default=6.0)
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
    """n pictures' syntax and their two reference pictures (content seeds per stream)."""
    pics, refs = [], []
    for i in range(n):
        seed = seed0 + 97 * i
        pics.append(hb.Picture(hb.default_cfg(w, h, seed, poc=8, **PICTURE_CFG)))
        refs.append([hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)])
    return pics, refs


def algorithmic_bytes(hb, pic):
    """Algorithmic HBM bytes per stage of one picture (reads + writes the stage must do)."""
    import numpy as np
    s = pic.syn
    W, H = s.params.width, s.params.height
    npu, ntu = s.num_pus, s.num_tus
    pu = np.ctypeslib.as_array(C.cast(s.pus, C.POINTER(C.c_uint8)), (npu * 20,)).view(
        np.dtype([("x", "<u2"), ("y", "<u2"), ("w", "u1"), ("h", "u1"), ("r", "i1", 2), ("mv", "<i2", 4),
                  ("wp", "<i2"), ("pad", "<u2")]))
    pw, ph = pu["w"].astype(np.int64), pu["h"].astype(np.int64)
    lists = (pu["r"] >= 0).sum(axis=1)
    mc_read = int((lists * ((pw + 7) * (ph + 7) + 2 * (pw // 2 + 3) * (ph // 2 + 3))).sum())
    mc_write = int((pw * ph * 3 // 2).sum())
    tu = np.ctypeslib.as_array(C.cast(s.tus, C.POINTER(C.c_uint8)), (ntu * 16,)).view(
        np.dtype([("x", "<u2"), ("y", "<u2"), ("l", "u1"), ("c", "u1"), ("qp", "u1"), ("f", "u1"), ("m", "u1"),
                  ("r", "u1", 3), ("off", "<u4")]))
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

def cpu_run(checker, pics, refs, n_pictures, threads):
    """Reconstruct n_pictures (round robin over the generated ones) on host threads."""
    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda i: checker.reconstruct_picture(pics[i % len(pics)], refs[i % len(pics)]),
                    range(n_pictures)))
    return time.perf_counter() - t0


def cpu_checker():
    import oracle
    if oracle.ref_available():
        return oracle.ref(), "reference"
    return oracle.port(), "port"


def run_reference(args, hb, rank, world):
    if rank != 0:
        return None
    pics, refs = make_streams(hb, args.batch, args.width, args.height, 1000)
    checker, kind = cpu_checker()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_run(checker, pics, refs, args.batch, threads)
    times = [cpu_run(checker, pics, refs, args.batch, threads) for _ in range(args.steps)]
    total = sum(times)
    value = args.batch * args.steps / total
    line = {"metric": METRIC, "value": round(value, 3), "unit": "frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * total / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32",
            "data": "synthetic (seeded P/B picture syntax and sinusoid references)", "impl": "reference",
            "config": {"workload": f"{args.width}x{args.height} 4:2:0 8-bit P/B picture reconstruction "
                                   f"(MC + residual + intra + deblocking + SAO), {args.batch} pictures per step",
                       "batch": args.batch, "parallelism": f"{threads} host threads, one picture per thread"},
            "cpu_baseline": {"value": round(value, 3), "unit": "frames/s", "cores": threads, "kind": kind,
                             "sample": f"{args.batch} pictures per step x {args.steps} steps"},
            "e2e": {"value": round(value, 3), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


# --------------------------------------------------------------------------- GPU arm

import ctypes as C  # noqa: E402


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
    W, H, B = args.width, args.height, args.batch
    slots = [2] * B
    import oracle
    check = oracle.port()

    def build_group(seed0, verify):
        """B streams with their two reference pictures in HBM and one prepared P/B
        picture each; verify: every picture bit-exact against the oracle first."""
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
        for i in range(B if verify else 0):
            got = g_streams[i].download(2)
            want = check.reconstruct_picture(g_pics[i], g_refs[i])
            if not np.array_equal(got, want):
                raise SystemExit(f"bench: picture {i} differs from the oracle in {int((got != want).sum())} samples")
        return g_pics, g_refs, g_streams, g_jobs

    # replicas: each rank reconstructs its own streams (different seeds), no collective.
    # Two groups of B streams: the served form alternates their batches over two lanes.
    verify = args.steps > 0 and not args.profile_only
    pics, refs, streams, jobs = build_group(rank_seed0(rank), verify)
    groups = [jobs]
    grp_pics, grp_streams = [pics], [streams]
    if not args.profile_only:
        pics_b, _, streams_b, jobs_b = build_group(rank_seed0(rank) + 50000, verify)
        groups.append(jobs_b)
        grp_pics.append(pics_b)
        grp_streams.append(streams_b)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def rank_max(x):
        return max_over_ranks(x, world, dev)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        ctx.sync()
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        step_ms = []
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        l0 = ctx.launches
        with torch.cuda.stream(stream):
            ev0.record(stream)
            evs[0].record(stream)
            for k in range(steps):
                fn()
                evs[k + 1].record(stream)
            ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1)
        step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
        return rank_max(ms), step_ms, ctx.launches - l0

    if args.profile_only:
        for _ in range(max(1, args.steps)):
            hb.batch_launch(jobs, slots)
        ctx.sync()
        return None

    # served form: batch k of B pictures goes to lane k % 2 (group k % 2), so consecutive
    # batches overlap on the device; timed from an event that both lanes wait for to the
    # later of the lanes' last events
    lanes = [hb.Lane(ctx), hb.Lane(ctx)]
    lane_st = [torch.cuda.ExternalStream(ln.cuda_stream, device=dev) for ln in lanes]

    def timed_served(steps, warmup):
        for k in range(warmup):
            lanes[k % 2].batch_launch(groups[k % 2], slots)
        for ln in lanes:
            ln.sync()
        ctx.sync()
        barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(lane_st[0])
        lane_st[1].wait_event(ev0)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        l0 = ctx.launches
        for k in range(steps):
            i = k % 2
            starts[k].record(lane_st[i])
            lanes[i].batch_launch(groups[i], slots)
            ends[k].record(lane_st[i])
        for ln in lanes:
            ln.sync()
        torch.cuda.synchronize()
        barrier()
        ms = max(ev0.elapsed_time(ends[steps - 1]), ev0.elapsed_time(ends[steps - 2]) if steps > 1 else 0.0)
        batch_ms = [starts[k].elapsed_time(ends[k]) for k in range(steps)]
        return rank_max(ms), batch_ms, ctx.launches - l0

    with ClockSampler(local) as clocks:
        served_ms, step_ms, launches = timed_served(args.steps, args.warmup)
    batched_steps = max(3, args.steps // 2)
    batched_ms, _, _ = timed(lambda: hb.batch_launch(jobs, slots), batched_steps, args.warmup)
    plain_steps = max(3, args.steps // 4)
    plain_ms, _, plain_launches = timed(lambda: [j.launch(2) for j in jobs], plain_steps, args.warmup)

    # stage profile (separate pass; events between stages)
    ctx.profile(True)
    prof_steps = max(3, args.steps // 4)
    for _ in range(prof_steps):
        hb.batch_launch(jobs, slots)
    stages = ctx.profile_read()
    ctx.profile(False)

    # end to end through the C ABI from host memory, pipelined over the two lanes: step k
    # prepares its B pictures on the host workers (records packed into pinned memory and
    # copied host->device: hevcgpu_jobs_prepare), launches them on lane k % 2 and queues the
    # copies of its frames into pinned host frame buffers behind them
    # (hevcgpu_lane_slots_download_async); the frames of step k are waited for
    # (hevcgpu_lane_wait) when their buffers come round again at step k + 2, and at the end
    frame_bytes = hb.i420_size(W, H)
    out_host = [[torch.empty(frame_bytes, dtype=torch.uint8).pin_memory().numpy() for _ in range(B)]
                for _ in range(2)]
    h2d_bytes = 0

    def e2e_run(steps):
        nonlocal h2d_bytes
        tickets, held = [None, None], [[], []]
        for k in range(steps):
            i = k % 2
            if tickets[i] is not None:
                lanes[i].wait(tickets[i])
                for j in held[i]:
                    j.free()
            js = hb.prepare_batch(grp_streams[i], grp_pics[i])
            h2d_bytes = sum(j.upload_bytes for j in js)
            lanes[i].batch_launch(js, slots)
            tickets[i] = lanes[i].download_batch_async(grp_streams[i], slots, out_host[i])
            held[i] = js
        for i in range(2):
            if tickets[i] is not None:
                lanes[i].wait(tickets[i])
                for j in held[i]:
                    j.free()

    # the records in page-locked memory, where a recorder writing into hevcgpu_host_alloc
    # buffers keeps them: their upload needs no staging copy (set up outside the timing)
    for g_pics in grp_pics:
        for p in g_pics:
            p.pin()
    e2e_steps = max(4, args.steps // 5)
    e2e_run(2)
    barrier()
    t0 = time.perf_counter()
    e2e_run(e2e_steps)
    e2e_s = rank_max(time.perf_counter() - t0)
    d2h_bytes = B * frame_bytes

    value = job_rate(B * args.steps, world, served_ms / 1000.0)
    batched_value = job_rate(B * batched_steps, world, batched_ms / 1000.0)
    plain_value = job_rate(B * plain_steps, world, plain_ms / 1000.0)
    e2e_value = job_rate(B * e2e_steps, world, e2e_s)

    # roofline of the dominant stage
    import json as _json
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(_json.load(open(peaks_path))["hbm_gbs"]), "measured"
    alg = [algorithmic_bytes(hb, p) for p in pics]
    alg_sum = {k: sum(a[k] for a in alg) for k in alg[0]}
    stage_ms = {"mc": stages["mc"][0], "residual": stages["residual"][0], "intra": stages["intra"][0],
                "deblock": stages["deblock_v"][0] + stages["deblock_h"][0], "sao": stages["sao"][0]}
    per_stage = {}
    for k, ms in stage_ms.items():
        per_launch_ms = ms / prof_steps
        gbs = alg_sum[k] / (per_launch_ms / 1000.0) / 1e9 if per_launch_ms > 0 else 0.0
        per_stage[k] = {"ms_per_step": round(per_launch_ms, 4), "alg_bytes_per_step": alg_sum[k],
                        "GB/s": round(gbs, 1), "frac_of_hbm": round(gbs / peak, 4)}
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    # DRAM bytes (read + write) per launch of each stage's kernels, from one ncu capture of
    # this workload at 16 pictures per launch (profiles/kernels_pb16_1080p.md); scaled by
    # the pictures per launch when --batch differs (the traffic grows with the pictures).
    ncu_dram_16 = {"mc": 146.71e6, "residual": 170.51e6, "intra": 50.43e6, "deblock": 160.87e6, "sao": 68.79e6}
    traffic = ncu_dram_16[dom] * B / 16.0 if W == W_DEFAULT and H == H_DEFAULT else None

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        checker, kind = cpu_checker()
        threads = os.cpu_count() or 1
        # bounded sample: about 10 s of wall time on all host threads
        t_probe = cpu_run(checker, pics, refs, threads, threads)
        n = threads * max(1, int(10.0 / max(t_probe, 1e-3)))
        t = cpu_run(checker, pics, refs, n, threads)
        cpu = {"value": round(n / t, 3), "unit": "frames/s", "cores": threads, "kind": kind,
               "sample": f"{n} of the bench's {W}x{H} pictures on {threads} host threads ({t:.1f} s)"}

    clk = clocks.summary()
    step_sorted = sorted(step_ms)
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(served_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32", "data": "synthetic (seeded P/B picture "
        "syntax and sinusoid reference pictures; no public dataset)",
        "config": {"workload": f"{W}x{H} 4:2:0 8-bit P/B picture reconstruction (MC + residual + intra wavefront + "
                               f"deblocking + SAO), {B} streams per batched launch, batches alternating over 2 "
                               f"lanes (2 x {B} streams, consecutive batches overlap on the device)",
                   "global_batch": B * world, "streams_in_flight": 2 * B * world,
                   "parallelism": f"replicas x{world} (streams sharded, no collective)",
                   "l2": "inputs larger than L2 (2 x B streams x 4 HBM buffers)"},
        "batched": {"value": round(batched_value, 2), "unit": "frames/s",
                    "ms_per_step": round(batched_ms / batched_steps, 4),
                    "note": "the same batches on one queue, no overlap between consecutive batches"},
        "plain": {"value": round(plain_value, 2), "unit": "frames/s", "ms_per_picture": round(plain_ms / plain_steps / B, 4),
                  "gpu_launches_per_picture": round(plain_launches / plain_steps / B, 1)},
        "batched_over_plain": round(value / plain_value, 3),
        "frame_ms": {"p50": round(statistics.median(step_ms), 4),
                     "p99": round(step_sorted[min(len(step_sorted) - 1, int(0.99 * len(step_sorted)))], 4),
                     "note": "device time from a batch's start on its lane to its completion; every "
                             "picture of a batch completes with it"},
        "e2e": {"value": round(e2e_value, 2), "unit": "frames/s", "h2d_bytes_per_step": int(h2d_bytes),
                "d2h_bytes_per_step": int(d2h_bytes)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": per_stage[dom]["GB/s"], "peak": peak,
                     "unit": "GB/s", "frac": per_stage[dom]["frac_of_hbm"],
                     "traffic": None if traffic is None else int(traffic),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one capture",
                     "peak_source": peak_src},
        "stages": per_stage,
        "clocks": clk,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    if not args.no_serving and rank == 0 and W == W_DEFAULT and H == H_DEFAULT:
        # the serving workload: 64 streams of mixed resolutions, Poisson segment arrivals
        from hevc_b200 import serve
        sctx = hb.Context(local)   # a serving process owns its context
        pool = serve.PicturePool(hb, [(416, 240), (1280, 720), (1920, 1080), (3840, 2160)], pin=True)
        # an unmeasured 2 s run first: the first use of a context's pools and launch paths
        # in a process costs once what a long-running server pays at start-up
        serve.run_poisson(hb, sctx, seconds=2.0, n_streams=64, seed=5, lanes=4, pool=pool)
        res = serve.run_poisson(hb, sctx, seconds=args.serve_seconds, n_streams=64, seed=4, lanes=4, pool=pool)
        sctx.close()
        line["serving"] = {
            "workload": "64 live streams, 416x240 / 1280x720 / 1920x1080 / 3840x2160 in ratio 4:3:2:1, "
                        "30 or 60 fps, 2-second segments (I picture, then P/B) arriving as a Poisson process "
                        f"(seed 4) for {args.serve_seconds:g} s; 4 lanes, continuous batching",
            "frames": res["frames"], "frames_per_s": round(res["frames_per_s"], 1),
            "p50_ms": round(res["p50_ms"], 2), "p99_ms": round(res["p99_ms"], 2), "max_ms": round(res["max_ms"], 2),
            "steady_p50_ms": round(res["steady_p50_ms"], 2), "steady_p99_ms": round(res["steady_p99_ms"], 2),
            "steady": "frames released after the first 2 s, when every stream's first segment (and its "
                      "I picture) has arrived",
            "latency": "device completion of the picture's batch minus the picture's live release time "
                       "(segment start + i / fps); records prepared on host workers, CABAC not included; "
                       "measured after an unmeasured 2 s warm-up run on the same context"}
    for ln in lanes:
        ln.close()
    for st in streams:
        st.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return line if rank == 0 else None


def main():
    args = parse()
    rank, world, local = dist_env()
    import __graft_entry__ as ge
    hb = ge.load_package()
    if args.impl == "reference":
        line = run_reference(args, hb, rank, world)
    else:
        line = run_ours(args, hb, rank, world, local)
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
