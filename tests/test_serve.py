"""Serving loop (hevc_b200.serve): continuous batching over lanes gives every stream the
bytes it gets decoded alone, and admission holds the HBM budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_streams_match_streams_decoded_alone(hb, gpu_ctx):
    from hevc_b200 import serve
    res = [(208, 120), (416, 240), (320, 176)]
    pool = serve.PicturePool(hb, res, variants=2)
    srv = serve.Server(hb, gpu_ctx, pool, lanes=2, max_batch=8)
    srv.start_clock(lambda: 0.0)
    specs = [(0, 208, 120), (1, 416, 240), (2, 320, 176), (3, 208, 120), (4, 416, 240)]
    segments = {sid: [7] for sid, _, _ in specs}
    segments[0] = [4, 5]          # two segments: a second I picture mid-stream
    for sid, w, h in specs:
        assert srv.admit(sid, w, h, fps=1000, variant=sid)
        t = 0.0
        for n in segments[sid]:
            srv.add_segment(sid, t, n)
            t += n / 1000.0
    latencies = []
    while srv.pending():
        latencies += srv.poll(1e9)    # every picture released
    srv.drain()
    assert len(latencies) == sum(sum(v) for v in segments.values())
    served = {sid: [srv.streams[sid].st.download(s) for s in range(serve.SLOTS)] for sid, _, _ in specs}
    srv.close()

    for sid, w, h in specs:
        st = gpu_ctx.open_stream(w, h, serve.SLOTS)
        for slot in range(1, serve.SLOTS):
            st.upload(slot, hb.content(w, h, srv.content_seed + 1000 * sid + slot))
        n = 0
        for seg in segments[sid]:
            for i in range(seg):
                job = st.prepare(pool.picture(w, h, i, n, sid))
                job.launch(n % serve.SLOTS)
                st.sync()
                job.free()
                n += 1
        for slot in range(serve.SLOTS):
            got = st.download(slot)
            assert np.array_equal(got, served[sid][slot]), (sid, slot)
        st.close()


def test_admission_holds_the_budget(hb):
    from hevc_b200 import serve
    ctx = hb.Context(0)
    pool = serve.PicturePool(hb, [(416, 240)], variants=1)
    frame = hb.i420_size(416, 240)
    # room for two streams' DPB + work buffers; DPBs alone (3 frames each) let a third in
    srv = serve.Server(hb, ctx, pool, lanes=1, budget_bytes=2 * (serve.SLOTS + 4) * frame)
    admitted = [srv.admit(sid, 416, 240, 30) for sid in range(4)]
    assert admitted[0] and admitted[1] and not admitted[3]
    assert ctx.bytes_in_use() <= srv.budget
    srv.close()
    ctx.close()
