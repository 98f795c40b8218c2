"""Multi-GPU replica path of bench.py, on CPU: two gloo ranks.

With N > 1 GPUs each rank reconstructs its own streams (the work shards by stream; there
is no data-path collective).  The host logic that makes that a whole-job number is tested
here without a GPU: ranks draw distinct streams, the timed region's length is the max
over ranks, the whole-job rate counts every rank's frames, and the reference arm runs on
rank 0 only."""
import datetime
import hashlib
import multiprocessing as mp
import os
import socket
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import __graft_entry__ as ge
        hb = ge.load_package()
        # distinct streams per rank
        pics, _ = bench.make_streams(hb, 2, 64, 64, bench.rank_seed0(rank))
        import ctypes
        h = hashlib.md5()
        for p in pics:
            h.update(ctypes.string_at(p.syn.tus, 16 * p.syn.num_tus))   # the TU records
        digests = [None] * world
        dist.all_gather_object(digests, h.hexdigest())
        # max over ranks of a per-rank time, and the whole-job rate
        local_s = 0.25 * (rank + 1)
        slowest = bench.max_over_ranks(local_s, world, torch.device("cpu"))
        rate = bench.job_rate(16 * 10, world, slowest)

        class Args:
            batch, steps, warmup, width, height, gpus, streams, gop = 2, 1, 0, 64, 64, world, 2, 3
        ref_line = bench.run_reference(Args, hb, rank, world) if rank != 0 else "rank0"
        out.put((rank, digests, slowest, rate, ref_line))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_streams_and_take_the_max():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r = q.get(timeout=240)
        results[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, digests, slowest, rate, ref_line in results.values():
        assert len(set(digests)) == world          # no two ranks reconstruct the same streams
        assert slowest == 0.25 * world             # the slowest rank's time, seen by every rank
        assert abs(rate - 16 * 10 * world / slowest) < 1e-9
        if rank != 0:
            assert ref_line is None                # the reference arm runs and prints on rank 0 only
