"""GPU parity: every stage of the CUDA back end, called through the C ABI, is bit-exact
against the oracle and against the reference's golden digests."""
import numpy as np
import pytest

import cases
from test_oracle import PCM_CASES, RESIDUAL_EDIT_CASES, _edit_blocks, with_filter_edits, with_residual_edits

pytestmark = pytest.mark.gpu


def _diff(a, b):
    return int((a != b).sum())


@pytest.mark.parametrize("name", list(cases.CASES))
def test_gpu_matches_reference_digests(hb, gpu_ctx, port, golden, name):
    case = cases.CASES[name]
    inp = cases.build_inputs(hb, case)
    got = cases.run_case(gpu_ctx, case, inp)
    want = cases.run_case(port, case, inp)
    assert _diff(got, want) == 0
    assert cases.digest(hb, case, got) == golden[name]["md5"]


@pytest.mark.parametrize("seed,opts", [(21, dict(tskip=True)), (22, dict(big=True, qp=(40, 51))),
                                       (23, dict(big=True, qp=(0, 10))), (24, dict(qp=(0, 51)))])
def test_gpu_blocks_edge_levels(hb, gpu_ctx, port, seed, opts):
    tus, n, coeffs, pred = _edit_blocks(hb, 600, seed, **opts)
    assert _diff(gpu_ctx.residual_blocks(tus, n, coeffs, pred), port.residual_blocks(tus, n, coeffs, pred)) == 0


@pytest.mark.parametrize("seed,opts", [(25, dict()), (26, dict(big=True)), (27, dict(tskip=True, big=True)),
                                       (28, dict(big=True, qp=(45, 51)))])
def test_gpu_blocks_scaled(hb, gpu_ctx, port, seed, opts):
    tus, n, coeffs, pred = _edit_blocks(hb, 800, seed, **opts)
    cases.mix_blocks(hb, tus, n, seed, qp=None if "qp" in opts else (0, 51))
    sl = hb.scaling(seed)
    got = gpu_ctx.residual_blocks(tus, n, coeffs, pred, sl)
    assert _diff(got, port.residual_blocks(tus, n, coeffs, pred, sl)) == 0
    assert _diff(gpu_ctx.residual_blocks(tus, n, coeffs, pred), port.residual_blocks(tus, n, coeffs, pred)) == 0


def test_gpu_blocks_empty(hb, gpu_ctx):
    tus, n, coeffs, pred = hb.blocks(0, 1)
    assert gpu_ctx.residual_blocks(tus, 0, coeffs, pred).size == pred.size


@pytest.mark.parametrize("seed,w,h,kw", [(31, 176, 144, dict(p_intra=0.3)), (32, 64, 64, dict(slice_type=2)),
                                         (33, 136, 72, dict(p_intra=0.2, p_skip=0.5, p_merge=0.6)),
                                         (34, 256, 192, dict(p_intra=0.7, p_intra_nxn=1.0)),
                                         (35, 320, 128, dict(p_wp=0.6, mv_range=4096)),
                                         (36, 3840, 2160, dict(p_intra=0.1)),
                                         (37, 1280, 720, dict(slice_type=2, strong_intra_smoothing=0)),
                                         (38, 640, 360, dict(p_intra=0.4, scaling_lists=1)),
                                         (39, 1280, 720, dict(slice_type=2, scaling_lists=1)),
                                         (40, 1920, 1080, dict(log2_ctb=4, p_intra=0.3)),
                                         (44, 1920, 1080, dict(log2_ctb=4, slice_type=2)),
                                         (45, 1280, 720, dict(log2_ctb=5, p_intra=0.5, p_intra_nxn=1.0)),
                                         (46, 1920, 1080, dict(tile_cols=5, tile_rows=3, log2_ctb=4, slice_type=2,
                                                               no_lf_across_tiles=1)),
                                         (47, 1280, 720, dict(tile_cols=4, tile_rows=2, p_intra=0.4)),
                                         (91, 320, 192, dict(slice_type=1, p_intra=0.2, p_wp=0.4)),
                                         (92, 256, 128, dict(num_refs=1, p_intra=0.2)),
                                         (94, 1920, 1080, dict(slice_type=1, p_wp=0.3))])
def test_gpu_pictures(hb, gpu_ctx, port, seed, w, h, kw):
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert _diff(gpu_ctx.reconstruct_picture(pic, refs), port.reconstruct_picture(pic, refs)) == 0


@pytest.mark.parametrize("seed,w,h,kw,params", RESIDUAL_EDIT_CASES + [(75, 1920, 1080, dict(p_intra=0.3), {})])
def test_gpu_bypass_tskip_qp_offsets(hb, gpu_ctx, port, seed, w, h, kw, params):
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    assert min(with_residual_edits(hb, pic, seed)) > 0
    for k, v in params.items():
        setattr(pic.syn.params, k, v)
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert _diff(gpu_ctx.reconstruct_picture(pic, refs), port.reconstruct_picture(pic, refs)) == 0


@pytest.mark.parametrize("seed,w,h,kw,lf_off", PCM_CASES + [(85, 1920, 1080, dict(p_intra=0.3, p_pcm=0.3), 1)])
def test_gpu_pcm(hb, gpu_ctx, port, seed, w, h, kw, lf_off):
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    pic.syn.params.pcm_loop_filter_disabled = lf_off
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert _diff(gpu_ctx.reconstruct_picture(pic, refs), port.reconstruct_picture(pic, refs)) == 0


@pytest.mark.parametrize("seed,w,h", [(41, 320, 192), (42, 200, 136), (43, 1920, 1080)])
def test_gpu_filters_with_slices_pcm_bypass(hb, gpu_ctx, port, seed, w, h):
    pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.FILTERS))
    keep = with_filter_edits(hb, pic, seed)
    src = hb.content(w, h, seed)
    for db, sao in [(True, True), (True, False), (False, True)]:
        assert _diff(gpu_ctx.loop_filter(pic, src, db, sao), port.loop_filter(pic, src, db, sao)) == 0, (db, sao)
    del keep


def test_dpb_jobs_plain_and_batched(hb, gpu_ctx, port):
    """Pictures of three streams of different sizes through the DPB API: plain launches
    and one batched launch give the oracle's pictures, and relaunching a prepared job
    reproduces the same output."""
    specs = [(416, 240, 51), (1920, 1080, 52), (208, 120, 53)]
    streams, jobs, want, pics = [], [], [], []
    for (w, h, seed) in specs:
        st = gpu_ctx.open_stream(w, h, 3)
        refs = [hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)]
        st.upload(0, refs[0])
        st.upload(1, refs[1])
        pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.PICTURE))
        pics.append(pic)
        want.append(port.reconstruct_picture(pic, refs))
        streams.append(st)
        jobs.append(st.prepare(pic))
    for st, job, wnt in zip(streams, jobs, want):
        job.launch(2)
        st.sync()
        assert _diff(st.download(2), wnt) == 0
        job.launch(2)
        st.sync()
        assert _diff(st.download(2), wnt) == 0
    # batched: clear the destinations first
    for st in streams:
        st.upload(2, np.zeros(hb.i420_size(st.width, st.height), np.uint8))
    hb.batch_launch(jobs, [2, 2, 2])
    gpu_ctx.sync()
    for st, wnt in zip(streams, want):
        assert _diff(st.download(2), wnt) == 0


def test_gop_through_a_lane_with_pending_downloads(hb, gpu_ctx, port):
    """A GOP (an I picture, then P/B pictures predicted from the two before them, over a
    ring of 3 DPB slots) through one lane, prepared from host records two positions at a
    time as the bench's end-to-end loop does, every picture downloaded asynchronously and
    nothing waited for until the end: picture n + 3 rewrites the slot whose download of
    picture n may still be pending, so it must wait for those copies on the device."""
    import torch
    import bench
    w, h, g, frames = 416, 240, 2, 7
    gop = bench.make_gop(hb, g, w, h, 4242)
    sts = []
    for s in gop:
        st = gpu_ctx.open_stream(w, h, 3)
        for k in range(3):
            st.upload(k, s[2][k])
        sts.append(st)
    want = []
    for s in gop:   # the oracle's chain
        dpb, outs = list(s[2]), []
        for n in range(frames):
            dpb[n % 3] = port.reconstruct_picture(bench.gop_picture(s, n), dpb)
            outs.append(dpb[n % 3])
        want.append(outs)
    lane = hb.Lane(gpu_ctx)
    size = hb.i420_size(w, h)
    got = [[torch.empty(size, dtype=torch.uint8).pin_memory().numpy() for _ in range(g)] for _ in range(frames)]
    for s in gop:   # page-locked records, prepared without waiting for their copies
        for pic in [s[0]] + s[1]:
            pic.pin()
    tickets, jobs = [], []
    for n0 in range(0, frames, 2):
        ns = [n for n in (n0, n0 + 1) if n < frames]
        js = hb.prepare_batch(sts * len(ns), [bench.gop_picture(s, n) for n in ns for s in gop], wait_uploads=False)
        for q, n in enumerate(ns):
            lane.batch_launch(js[q * g:(q + 1) * g], [n % 3] * g)
            tickets.append(lane.download_batch_async(sts, [n % 3] * g, got[n]))
        jobs += js
    for t in tickets:
        lane.wait(t)
    for n in range(frames):
        for i in range(g):
            assert _diff(got[n][i], want[i][n]) == 0, (n, i)
    for j in jobs:
        j.free()
    lane.close()


def test_prepare_async_then_overwrite_the_records(hb, gpu_ctx, port):
    """hevcgpu_jobs_prepare_async + hevcgpu_job_wait_uploaded: once the wait returns, the
    caller may overwrite its page-locked record arrays; the job keeps the picture it was
    prepared from."""
    w, h = 320, 192
    streams, pics, want = [], [], []
    for seed in (95, 96):
        st = gpu_ctx.open_stream(w, h, 3)
        refs = [hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)]
        st.upload(0, refs[0])
        st.upload(1, refs[1])
        pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.PICTURE))
        want.append(port.reconstruct_picture(pic, refs))
        pic.pin()
        streams.append(st)
        pics.append(pic)
    jobs = hb.prepare_batch(streams, pics, wait_uploads=False)
    for j, pic in zip(jobs, pics):
        j.wait_uploaded()
        s = pic.syn
        np.ctypeslib.as_array(s.coeffs, (s.num_coeffs,))[:] = 0   # the recorder reuses its buffers
        for k in range(s.num_pus):
            s.pus[k].mv[0][0] += 64
    hb.batch_launch(jobs, [2, 2])
    gpu_ctx.sync()
    for st, wnt in zip(streams, want):
        assert _diff(st.download(2), wnt) == 0
    for j in jobs:
        j.free()


def test_bounded_wait_times_out_and_the_context_recovers(hb, gpu_ctx, port):
    """The intra stage's cross-CTU waits are bounded: a wait for a level that nothing
    publishes (planted in the job's schedule on the host) gives up after about a second,
    the sync reports HEVCGPU_ETIMEOUT, and the context then decodes correctly again."""
    import time
    w, h, seed = 128, 64, 97
    st = gpu_ctx.open_stream(w, h, 3)
    refs = [hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)]
    st.upload(0, refs[0])
    st.upload(1, refs[1])
    pic = hb.Picture(hb.default_cfg(w, h, seed, **dict(cases.PICTURE, p_intra=0.5)))
    job = st.prepare(pic)
    job.plant_unmet_wait()
    t0 = time.perf_counter()
    job.launch(2)
    with pytest.raises(hb.HevcGpuError) as e:
        st.sync()
    waited = time.perf_counter() - t0
    assert e.value.code == hb.abi.HEVCGPU_ETIMEOUT
    assert 0.5 < waited < 30.0
    job.free()
    fresh = st.prepare(pic)
    fresh.launch(2)
    st.sync()
    assert _diff(st.download(2), port.reconstruct_picture(pic, refs)) == 0
    fresh.free()
    flat = hb.Picture(hb.default_cfg(w, h, seed, p_intra=0.0))
    j = st.prepare(flat)
    with pytest.raises(hb.HevcGpuError) as e:
        j.plant_unmet_wait()
    assert e.value.code == hb.abi.HEVCGPU_EINVAL
    j.free()


def test_bounded_wait_gives_up_once_on_a_large_picture(hb, gpu_ctx, port):
    """A 1080p all-intra picture with 16x16 CTBs (8160 CTUs, many more than the launch holds
    resident): when the first CTU's wait gives up, the CTUs that wait behind it, and the CTAs
    that start after it, see the status word and end at once instead of each running out a
    second of their own.  The context then decodes the picture correctly."""
    import time
    w, h, seed = 1920, 1080, 98
    st = gpu_ctx.open_stream(w, h, 3)
    pic = hb.Picture(hb.default_cfg(w, h, seed, slice_type=2, log2_ctb=4))
    job = st.prepare(pic)
    job.plant_unmet_wait()
    t0 = time.perf_counter()
    job.launch(2)
    with pytest.raises(hb.HevcGpuError) as e:
        st.sync()
    waited = time.perf_counter() - t0
    assert e.value.code == hb.abi.HEVCGPU_ETIMEOUT
    assert 0.5 < waited < 5.0
    job.free()
    fresh = st.prepare(pic)
    fresh.launch(2)
    st.sync()
    assert _diff(st.download(2), port.reconstruct_picture(pic, [])) == 0
    fresh.free()


def test_frame_output_cropped_16bit(hb, gpu_ctx, port):
    """hevcgpu_slot_download_frame gives the reconstructed picture inside the conformance
    window as 16-bit planes, as hevc_decoder_get_frame does (hevc_api.cpp:49-77)."""
    w, h, seed = 216, 136, 91
    st = gpu_ctx.open_stream(w, h, 3)
    refs = [hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)]
    st.upload(0, refs[0])
    st.upload(1, refs[1])
    pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.PICTURE))
    want = hb.split_i420(port.reconstruct_picture(pic, refs), w, h)
    job = st.prepare(pic)
    job.launch(2)
    st.sync()
    for crop, strides in [(None, (None, None)), ((2, 6, 4, 8), (None, None)), ((8, 0, 0, 2), (240, 130)),
                          ((0, 14, 6, 0), (202, 101))]:
        l, r, t, b = crop or (0, 0, 0, 0)
        got = st.download_frame(2, crop, *strides)
        for p, (g, full) in enumerate(zip(got, want)):
            sub = 2 if p else 1
            exp = full[t // sub: (h - b) // sub, l // sub: (w - r) // sub].astype(np.uint16)
            assert g.dtype == np.uint16 and g.shape == exp.shape, (crop, p)
            assert _diff(g, exp) == 0, (crop, p)
    for bad in [(1, 0, 0, 0), (0, 0, -2, 0), (108, 108, 0, 0), (0, 0, 70, 66)]:
        with pytest.raises(hb.HevcGpuError) as e:
            st.download_frame(2, bad)
        assert e.value.code == hb.abi.HEVCGPU_EINVAL
    job.free()


def test_slot_checksum_on_the_device(hb, gpu_ctx, port):
    """hevcgpu_slot_checksum gives the H.265 picture hash SEI checksum (D.3.19) of each plane of
    the frame hevcgpu_slot_download_frame hands out: equal to the checksum of the oracle's
    picture (no frame copy needed) and of the downloaded frame, with and without a
    conformance window, at a size with coordinates past 255 (the >> 8 terms of the mask)."""
    for w, h, seed in ((216, 136, 91), (1920, 1080, 4)):
        st = gpu_ctx.open_stream(w, h, 3)
        refs = [hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)]
        st.upload(0, refs[0])
        st.upload(1, refs[1])
        pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.PICTURE))
        want = hb.split_i420(port.reconstruct_picture(pic, refs), w, h)
        job = st.prepare(pic)
        job.launch(2)
        st.sync()
        for crop in (None, (2, 6, 4, 8), (0, 14, 6, 0), (8, 0, 0, 2)):
            l, r, t, b = crop or (0, 0, 0, 0)
            got = st.checksum(2, crop)
            exp = tuple(cases.picture_checksum(full[t // sub: (h - b) // sub, l // sub: (w - r) // sub])
                        for full, sub in zip(want, (1, 2, 2)))
            assert got == exp, (w, crop)
            assert got == tuple(cases.picture_checksum(pl) for pl in st.download_frame(2, crop)), (w, crop)
        for bad in [(1, 0, 0, 0), (0, 0, -2, 0), (w // 2, w // 2, 0, 0)]:
            with pytest.raises(hb.HevcGpuError) as e:
                st.checksum(2, bad)
            assert e.value.code == hb.abi.HEVCGPU_EINVAL
        job.free()


def test_batched_prepare_and_download(hb, gpu_ctx, port):
    """hevcgpu_jobs_prepare + hevcgpu_batch_launch + hevcgpu_slots_download over streams
    of mixed sizes give the oracle's pictures into pageable and pinned host buffers; a
    failing picture makes the whole preparation fail with no job returned."""
    import torch
    specs = [(416, 240, 81), (1280, 720, 82), (208, 120, 83), (640, 360, 84), (1920, 1080, 85)]
    streams, pics, want = [], [], []
    for (w, h, seed) in specs:
        st = gpu_ctx.open_stream(w, h, 3)
        refs = [hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)]
        st.upload(0, refs[0])
        st.upload(1, refs[1])
        pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.PICTURE))
        streams.append(st)
        pics.append(pic)
        want.append(port.reconstruct_picture(pic, refs))
    for rep in range(3):
        if rep == 2:   # records in page-locked memory: uploaded without the staging copy
            for pic in pics[::2]:
                pic.pin()
            for st in streams:
                st.upload(2, np.zeros(hb.i420_size(st.width, st.height), np.uint8))
        jobs = hb.prepare_batch(streams, pics)
        hb.batch_launch(jobs, [2] * len(jobs))
        if rep != 1:
            outs = hb.download_batch(streams, [2] * len(streams))
        else:   # pinned destinations take the copy directly
            outs = [torch.empty(hb.i420_size(st.width, st.height), dtype=torch.uint8).pin_memory().numpy()
                    for st in streams]
            hb.download_batch(streams, [2] * len(streams), outs)
        for got, wnt in zip(outs, want):
            assert _diff(got, wnt) == 0
        for j in jobs:
            j.free()
    bad = hb.Picture(hb.default_cfg(208, 120, 86, **cases.PICTURE))
    bad.syn.tus[0].x = 4000
    with pytest.raises(hb.HevcGpuError) as e:
        hb.prepare_batch([streams[2], streams[0]], [bad, pics[0]])
    assert e.value.code == hb.abi.HEVCGPU_EINVAL
    assert "picture 0" in str(e.value)


def test_lanes_alone_and_in_the_mix(hb, gpu_ctx, port):
    """Pictures of mixed sizes give the same bytes decoded alone (plain launch on the
    context) and decoded in overlapping batches on two lanes, round after round, and a
    job moved from one lane to the other reproduces them again."""
    specs = [(416, 240, 91, cases.PICTURE), (1280, 720, 92, cases.PICTURE), (1920, 1080, 93, cases.PICTURE),
             (640, 360, 94, dict(slice_type=2)), (208, 120, 95, cases.INTRA_HEAVY), (1920, 1080, 96, cases.PICTURE)]
    streams, jobs, alone = [], [], []
    for (w, h, seed, kw) in specs:
        st = gpu_ctx.open_stream(w, h, 3)
        refs = [hb.content(w, h, seed + 1), hb.content(w, h, seed + 2)]
        st.upload(0, refs[0])
        st.upload(1, refs[1])
        pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
        job = st.prepare(pic)
        job.launch(2)
        st.sync()
        got = st.download(2)
        assert _diff(got, port.reconstruct_picture(pic, refs)) == 0
        streams.append(st)
        jobs.append(job)
        alone.append(got)
    lanes = [hb.Lane(gpu_ctx), hb.Lane(gpu_ctx)]
    groups = [[0, 2, 4], [1, 3, 5]]
    for st in streams:
        st.upload(2, np.zeros(hb.i420_size(st.width, st.height), np.uint8))
    for _ in range(3):
        for lane, g in zip(lanes, groups):
            lane.batch_launch([jobs[i] for i in g], [2] * len(g))
    for lane in lanes:
        lane.sync()
    for st, want in zip(streams, alone):
        assert _diff(st.download(2), want) == 0
    # job 0 last ran on lane 0; run it on lane 1 into a cleared slot
    streams[0].upload(2, np.zeros(hb.i420_size(streams[0].width, streams[0].height), np.uint8))
    lanes[1].batch_launch([jobs[0]], [2])
    lanes[1].sync()
    assert _diff(streams[0].download(2), alone[0]) == 0
    # a lane's download is ordered after its own batches, without a sync first
    for st in streams:
        st.upload(2, np.zeros(hb.i420_size(st.width, st.height), np.uint8))
    lanes[0].batch_launch([jobs[i] for i in groups[0]], [2] * 3)
    outs = [np.empty(hb.i420_size(streams[i].width, streams[i].height), np.uint8) for i in groups[0]]
    lanes[0].download_batch([streams[i] for i in groups[0]], [2] * 3, outs)
    for i, got in zip(groups[0], outs):
        assert _diff(got, alone[i]) == 0
    # asynchronous downloads into pinned buffers: queued behind the lane's batch, complete
    # after the wait on their ticket, two in flight on the two lanes at once
    import torch
    for st in streams:
        st.upload(2, np.zeros(hb.i420_size(st.width, st.height), np.uint8))
    pinned = [torch.empty(hb.i420_size(st.width, st.height), dtype=torch.uint8).pin_memory().numpy()
              for st in streams]
    tickets = []
    for lane, g in zip(lanes, groups):
        lane.batch_launch([jobs[i] for i in g], [2] * len(g))
        tickets.append(lane.download_batch_async([streams[i] for i in g], [2] * len(g), [pinned[i] for i in g]))
    for lane, t in zip(lanes, tickets):
        lane.wait(t)
    for got, want in zip(pinned, alone):
        assert _diff(got, want) == 0
    # a pageable destination is refused: the asynchronous copies write their destinations directly
    with pytest.raises(hb.HevcGpuError) as e:
        lanes[0].download_batch_async([streams[0]], [2], [np.empty_like(alone[0])])
    assert e.value.code == hb.abi.HEVCGPU_EINVAL
    for lane in lanes:
        lane.close()


def test_picture_decode_end_to_end(hb, gpu_ctx, port):
    w, h = 640, 360
    st = gpu_ctx.open_stream(w, h, 3)
    refs = [hb.content(w, h, 71), hb.content(w, h, 72)]
    st.upload(0, refs[0])
    st.upload(1, refs[1])
    pic = hb.Picture(hb.default_cfg(w, h, 70, **cases.PICTURE))
    st.decode(pic, 2)
    assert _diff(st.download(2), port.reconstruct_picture(pic, refs)) == 0


def test_invalid_records_are_refused(hb, gpu_ctx):
    w, h = 128, 64
    pic = hb.Picture(hb.default_cfg(w, h, 5, **cases.PICTURE))
    refs = [hb.content(w, h, 1), hb.content(w, h, 2)]
    s = pic.syn
    t0 = s.tus[0]
    old = (t0.x, t0.coeff_offset)
    s.tus[0].x = 4000
    with pytest.raises(hb.HevcGpuError) as e:
        gpu_ctx.reconstruct_picture(pic, refs)
    assert e.value.code == hb.abi.HEVCGPU_EINVAL
    s.tus[0].x = old[0]
    flags = s.tus[0].flags
    s.tus[0].flags = hb.abi.HEVC_TU_CODED | hb.abi.HEVC_TU_PCM   # PCM needs an intra TU
    with pytest.raises(hb.HevcGpuError) as e:
        gpu_ctx.reconstruct_picture(pic, refs)
    assert e.value.code == hb.abi.HEVCGPU_EINVAL and "PCM" in str(e.value)
    s.tus[0].flags = flags
    s.pus[0].ref_idx[0] = 9
    with pytest.raises(hb.HevcGpuError):
        gpu_ctx.reconstruct_picture(pic, refs)
    st = gpu_ctx.open_stream(w, h, 2)
    with pytest.raises(hb.HevcGpuError):
        st.upload(5, refs[0])
    with pytest.raises(hb.HevcGpuError):
        gpu_ctx.open_stream(100, 60, 2)   # not a multiple of 8


def test_budget_admission(hb, gpu_ctx):
    from hevc_b200 import HevcGpuError
    ctx = hb.Context(0)
    ctx.set_budget(8 << 20)
    with pytest.raises(HevcGpuError) as e:
        ctx.open_stream(1920, 1080, 4)   # 4 x 3.1 MB > 8 MB
    assert e.value.code == hb.abi.HEVCGPU_ENOMEM
    st = ctx.open_stream(416, 240, 2)
    assert ctx.bytes_in_use() <= 8 << 20
    st.close()
    ctx.close()


def test_gpu_reconstructs_recorded_real_streams(hb, gpu_ctx):
    """The records of the reference's own conformance streams (tests/golden/real/, recorded
    inside privaloops/hevc.js by oracle/recorder.cpp) through the DPB API: every picture,
    predicted from the GPU's own earlier pictures in its stream's slots, has the MD5 of the
    picture the reference decoded."""
    import hashlib
    import json
    import os
    import sys
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, golden)
    import real_streams
    want = json.load(open(os.path.join(golden, "real_streams.json")))["streams"]
    for name in sorted(want):
        pics = real_streams.load(hb.abi, os.path.join(real_streams.DIR, name + ".hrec.xz"))
        assert len(pics) <= 16   # one slot per picture: params.ref_slot (decode indices) are the slots
        st = gpu_ctx.open_stream(pics[0].width, pics[0].height, 16)
        for k, pic in enumerate(pics):
            job = st.prepare(pic)
            job.launch(k)
            st.sync()
            assert hashlib.md5(st.download(k).tobytes()).hexdigest() == want[name]["md5"][k], (name, k)
            job.free()
        st.close()


def test_gpu_full_gop_chain_1080p(hb, gpu_ctx, port):
    """Two streams of the bench's GOP workload (1920x1080, an I picture then 59 P/B pictures,
    each predicted from the two before it in a 3-slot DPB ring), batched as the bench runs
    them: every one of the 120 pictures equals the oracle's chain."""
    import bench
    gop = bench.make_gop(hb, 2, 1920, 1080, 4242)
    sts = []
    for _, _, init in gop:
        st = gpu_ctx.open_stream(1920, 1080, bench.SLOTS)
        for s in range(bench.SLOTS):
            st.upload(s, init[s])
        sts.append(st)
    jobs_i = [st.prepare(g[0]) for st, g in zip(sts, gop)]
    jobs_pb = [[st.prepare(g[1][ph]) for st, g in zip(sts, gop)] for ph in range(bench.SLOTS)]
    errs = bench.verify_gop_chain(hb, port, gop, sts, lambda n: jobs_i if n == 0 else jobs_pb[n % bench.SLOTS], 60)
    assert not errs, errs[:4]
