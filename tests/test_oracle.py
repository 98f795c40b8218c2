"""The CPU restatement (oracle/hevc_oracle.c) against privaloops/hevc.js.

Pinned two ways: against the committed golden digests that the reference's own
functions produced (tests/golden/make_golden.py), and — when the reference harness
oracle/_ref is built — directly against it on further seeds and edge cases.
"""
import ctypes as C

import numpy as np
import pytest

import cases


@pytest.mark.parametrize("name", list(cases.CASES))
def test_port_reproduces_reference_digests(hb, port, golden, name):
    case = cases.CASES[name]
    inp = cases.build_inputs(hb, case)
    out = cases.run_case(port, case, inp)
    assert cases.digest(hb, case, out) == golden[name]["md5"]


def test_filter_cases_realise_target_bs_mix(golden):
    # config 3 asks for Bs 0/1/2 drawn 0.5/0.3/0.2; the syntax realises it within 5 %
    h = golden["filters_1080p_s2"]["bs_histogram"]
    f = [x / sum(h) for x in h]
    assert abs(f[0] - 0.5) < 0.05 and abs(f[1] - 0.3) < 0.05 and abs(f[2] - 0.2) < 0.05


def _ref():
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference harness oracle/_ref not built (needs the reference tree at build time)")
    return oracle.ref()


def _edit_blocks(hb, n, seed, tskip=False, big=False, qp=None):
    tus, n, coeffs, pred = hb.blocks(n, seed)
    rng = np.random.default_rng(seed)
    for i in range(n):
        if tskip and tus[i].log2_size == 2 and rng.random() < 0.5:
            tus[i].flags |= hb.abi.HEVC_TU_TSKIP
        if qp is not None:
            tus[i].qp = int(rng.integers(qp[0], qp[1] + 1))
    if big:
        # levels near the int16 limits: exercises the reference's int64 product,
        # its narrowing to int and the int16 clips between the passes
        mask = rng.random(coeffs.size) < 0.3
        coeffs[mask] = rng.choice(np.array([-32768, -32767, 32767, -20000, 25000], np.int16), mask.sum())
    return tus, n, coeffs, pred


@pytest.mark.parametrize("seed,opts", [(21, dict(tskip=True)), (22, dict(big=True, qp=(40, 51))),
                                       (23, dict(big=True, qp=(0, 10))), (24, dict(qp=(0, 51)))])
def test_port_matches_reference_blocks(hb, port, seed, opts):
    ref = _ref()
    tus, n, coeffs, pred = _edit_blocks(hb, 600, seed, **opts)
    assert np.array_equal(port.residual_blocks(tus, n, coeffs, pred), ref.residual_blocks(tus, n, coeffs, pred))


@pytest.mark.parametrize("seed,w,h,kw", [(51, 176, 144, dict(log2_ctb=4, p_intra=0.3)),
                                         (52, 208, 120, dict(log2_ctb=5, p_intra=0.3)),
                                         (53, 128, 96, dict(log2_ctb=4, slice_type=2)),
                                         (54, 320, 192, dict(log2_ctb=5, p_intra=0.6, p_intra_nxn=1.0))])
def test_port_matches_reference_small_ctbs(hb, port, seed, w, h, kw):
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    assert pic.syn.params.log2_ctb == kw["log2_ctb"]
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert np.array_equal(port.reconstruct_picture(pic, refs), ref.reconstruct_picture(pic, refs))


@pytest.mark.parametrize("seed,w,h,kw", [(61, 320, 192, dict(tile_cols=3, tile_rows=2, p_intra=0.4)),
                                         (62, 320, 192, dict(tile_cols=2, tile_rows=2, p_intra=0.4, no_lf_across_tiles=1)),
                                         (63, 256, 128, dict(tile_cols=4, tile_rows=1, slice_type=2, no_lf_across_tiles=1,
                                                             log2_ctb=5)),
                                         (64, 416, 240, dict(tile_cols=3, tile_rows=3, p_intra=0.3, log2_ctb=4,
                                                             no_lf_across_tiles=1))])
def test_port_matches_reference_tiles(hb, port, seed, w, h, kw):
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    assert pic.syn.params.tiles_enabled == 1
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert np.array_equal(port.reconstruct_picture(pic, refs), ref.reconstruct_picture(pic, refs))


@pytest.mark.parametrize("seed,opts", [(25, dict()), (26, dict(big=True)), (27, dict(tskip=True, big=True))])
def test_port_matches_reference_scaled_blocks(hb, port, seed, opts):
    # scaling lists with factors up to 255: with levels near the int16 limits the
    # reference's int64 product overflows int before its clip, which the port narrows alike
    ref = _ref()
    tus, n, coeffs, pred = _edit_blocks(hb, 800, seed, **opts)
    cases.mix_blocks(hb, tus, n, seed)
    sl = hb.scaling(seed)
    got = port.residual_blocks(tus, n, coeffs, pred, sl)
    assert np.array_equal(got, ref.residual_blocks(tus, n, coeffs, pred, sl))
    assert not np.array_equal(got, port.residual_blocks(tus, n, coeffs, pred))


@pytest.mark.parametrize("seed,w,h,kw", [(41, 176, 144, dict(p_intra=0.3)), (42, 64, 64, dict(slice_type=2)),
                                         (43, 256, 192, dict(p_intra=0.6, p_intra_nxn=1.0))])
def test_port_matches_reference_scaled_pictures(hb, port, seed, w, h, kw):
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, scaling_lists=1, **kw))
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert np.array_equal(port.reconstruct_picture(pic, refs), ref.reconstruct_picture(pic, refs))


@pytest.mark.parametrize("seed,w,h,kw", [(31, 176, 144, dict(p_intra=0.3)), (32, 64, 64, dict(slice_type=2)),
                                         (33, 136, 72, dict(p_intra=0.2, p_skip=0.5, p_merge=0.6)),
                                         (34, 256, 192, dict(p_intra=0.7, p_intra_nxn=1.0)),
                                         (35, 320, 128, dict(p_wp=0.6, mv_range=4096)),
                                         (91, 320, 192, dict(slice_type=1, p_intra=0.2, p_wp=0.4)),
                                         (92, 256, 128, dict(num_refs=1, p_intra=0.2)),
                                         (93, 320, 192, dict(slice_type=1, num_refs=1, p_wp=0.5))])
def test_port_matches_reference_pictures(hb, port, seed, w, h, kw):
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert np.array_equal(port.reconstruct_picture(pic, refs), ref.reconstruct_picture(pic, refs))


def with_filter_edits(hb, pic, seed, slices=True, pcm_bypass=True):
    """Mutate a generated picture: PCM/bypass CUs, several slices with their own filter
    parameters (one with deblocking disabled, one not filtering across slices)."""
    syn = pic.syn
    p = syn.params
    rng = np.random.default_rng(seed)
    keep = {}
    if pcm_bypass:
        blk = np.ctypeslib.as_array(syn.blk, ((p.height // 4) * (p.width // 4),))
        n8w, n8h = p.width // 8, p.height // 8
        pick = rng.random((n8h, n8w)) < 0.08
        for (by, bx) in zip(*np.nonzero(pick)):
            bit = hb.abi.HEVC_BLK_PCM if rng.random() < 0.5 else hb.abi.HEVC_BLK_BYPASS
            for dy in range(2):
                for dx in range(2):
                    blk[(2 * by + dy) * (p.width // 4) + 2 * bx + dx] |= bit
        syn.params.pcm_loop_filter_disabled = 1
    if slices:
        ctb = 1 << p.log2_ctb
        wc, hc = (p.width + ctb - 1) // ctb, (p.height + ctb - 1) // ctb
        sl = np.ctypeslib.as_array(syn.ctb_slice, (wc * hc,))
        bounds = sorted(rng.choice(np.arange(1, wc * hc), size=3, replace=False))
        idx = np.zeros(wc * hc, np.uint8)
        for b in bounds:
            idx[b:] += 1
        sl[:] = idx
        arr = (hb.Slice * 4)()
        params = [(0, 0, 0, 1), (2, -2, 0, 0), (-3, 3, 1, 1), (1, 1, 0, 0)]
        for i, (b, t, dis, lf) in enumerate(params):
            arr[i].beta_offset_div2, arr[i].tc_offset_div2 = b, t
            arr[i].deblocking_disabled, arr[i].lf_across_slices = dis, lf
        keep["slices"] = arr
        syn.slices = C.cast(arr, C.POINTER(hb.Slice))
        syn.num_slices = 4
    return keep


def with_residual_edits(hb, pic, seed, p_bypass=0.1, p_tskip=0.5):
    """Mutate a generated picture: some CUs transquant-bypass (their TUs' levels are the
    residual, coding_tree.cpp:1302-1304, and the grid marks them, so that the filters leave
    their samples alone), and about half the coded 4x4 TUs of the others transform-skipped.
    Returns the numbers of bypass and transform-skip TUs made."""
    syn, p = pic.syn, pic.syn.params
    rng = np.random.default_rng(seed)
    cus = pic.ptr.contents
    gw, gh = p.width // 4, p.height // 4
    blk = np.ctypeslib.as_array(syn.blk, (gh * gw,))
    n_bypass = n_tskip = 0
    for i in range(cus.num_cus):
        cu = cus.cus[i]
        bypass = rng.random() < p_bypass
        for k in range(cu.first_tu, cu.first_tu + cu.num_tu):
            t = syn.tus[k]
            if bypass:
                t.flags |= hb.abi.HEVC_TU_BYPASS
                n_bypass += 1
            elif (t.flags & hb.abi.HEVC_TU_CODED) and t.log2_size == 2 and rng.random() < p_tskip:
                t.flags |= hb.abi.HEVC_TU_TSKIP
                n_tskip += 1
        if bypass:
            n = 1 << cu.log2_size
            for y in range(cu.y // 4, min((cu.y + n) // 4, gh)):
                blk[y * gw + cu.x // 4: y * gw + min((cu.x + n) // 4, gw)] |= hb.abi.HEVC_BLK_BYPASS
    return n_bypass, n_tskip


# pictures with bypass and transform-skip TUs, chroma QP offsets, intra smoothing off
RESIDUAL_EDIT_CASES = [(71, 320, 192, dict(p_intra=0.4), {}),
                       (72, 256, 128, dict(slice_type=2), {}),
                       (73, 320, 192, dict(p_intra=0.3, cb_qp_offset=5, cr_qp_offset=-4), {}),
                       (74, 256, 192, dict(p_intra=0.6, p_intra_nxn=1.0), {"intra_smoothing_disabled": 1})]


@pytest.mark.parametrize("seed,w,h,kw,params", RESIDUAL_EDIT_CASES)
def test_port_matches_reference_bypass_tskip_qp_offsets(hb, port, seed, w, h, kw, params):
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    assert min(with_residual_edits(hb, pic, seed)) > 0
    for k, v in params.items():
        setattr(pic.syn.params, k, v)
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    got = port.reconstruct_picture(pic, refs)
    assert np.array_equal(got, ref.reconstruct_picture(pic, refs))


@pytest.mark.parametrize("seed,w,h,kw", [
    (101, 320, 192, dict(qp_min=0, qp_max=51, p_intra=0.3, beta_offset_div2=6, tc_offset_div2=6)),
    (102, 320, 192, dict(qp_min=0, qp_max=51, p_intra=0.3, beta_offset_div2=-6, tc_offset_div2=-6)),
    (103, 256, 128, dict(qp_min=45, qp_max=51, slice_type=2, tc_offset_div2=6, cb_qp_offset=12, cr_qp_offset=-12)),
    (104, 256, 128, dict(qp_min=0, qp_max=4, p_intra=0.5, cb_qp_offset=-12, cr_qp_offset=12))])
def test_port_matches_reference_extreme_qps_and_offsets(hb, port, seed, w, h, kw):
    # the ends of the beta / tC / chroma QP tables (clipped indices) in whole pictures
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert np.array_equal(port.reconstruct_picture(pic, refs), ref.reconstruct_picture(pic, refs))


# PCM CUs (HEVC_TU_PCM: the levels are the samples), with and without pcm_loop_filter_disabled
PCM_CASES = [(81, 320, 192, dict(p_intra=0.5, p_pcm=0.3), 0), (82, 320, 192, dict(p_intra=0.5, p_pcm=0.3), 1),
             (83, 256, 128, dict(slice_type=2, p_pcm=0.4), 1), (84, 208, 120, dict(slice_type=2, p_pcm=0.5, log2_ctb=4), 0)]


@pytest.mark.parametrize("seed,w,h,kw,lf_off", PCM_CASES)
def test_port_matches_reference_pcm(hb, port, seed, w, h, kw, lf_off):
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, **kw))
    pic.syn.params.pcm_loop_filter_disabled = lf_off
    assert any(pic.syn.tus[i].flags & hb.abi.HEVC_TU_PCM for i in range(pic.syn.num_tus))
    refs = [hb.content(w, h, seed + 1000), hb.content(w, h, seed + 2000)]
    assert np.array_equal(port.reconstruct_picture(pic, refs), ref.reconstruct_picture(pic, refs))


@pytest.mark.parametrize("seed,w,h", [(41, 320, 192), (42, 200, 136)])
def test_port_matches_reference_filters_with_slices_pcm_bypass(hb, port, seed, w, h):
    ref = _ref()
    pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.FILTERS))
    keep = with_filter_edits(hb, pic, seed)
    src = hb.content(w, h, seed)
    for db, sao in [(True, True), (True, False), (False, True)]:
        a = port.loop_filter(pic, src, db, sao)
        b = ref.loop_filter(pic, src, db, sao)
        assert np.array_equal(a, b), (db, sao, int((a != b).sum()))
    del keep
