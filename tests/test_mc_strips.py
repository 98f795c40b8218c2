"""The motion-compensation work lists the back end builds (hevcgpu_mc_strips), on the CPU:
every PU's luma area, and its area in each chroma plane, is covered by its strips exactly
once (so k_mc predicts every inter sample once, interpolation.cpp:306-411 per PU), and
each list is ordered with bi-predicted strips first and, within one prediction kind and
window class, taller strips first (the order that keeps the threads of a warp on one path)."""
import numpy as np
import pytest

import cases

CONFIGS = {
    "P/B 1920x1080": dict(w=1920, h=1080, seed=1011, cfg=dict(cases.PICTURE, poc=8)),
    "P/B 416x240, 32x32 CTBs": dict(w=416, h=240, seed=17, cfg=dict(cases.PICTURE, poc=8, log2_ctb=5)),
    "P/B 72x40": dict(w=72, h=40, seed=12, cfg=dict(cases.PICTURE, poc=8, p_intra=0.4)),
    "B 208x120, 16x16 CTBs": dict(w=208, h=120, seed=31, cfg=dict(cases.PICTURE, poc=8, log2_ctb=4, p_bi=0.9)),
}


def decode(item, chroma):
    pu = item & 0xFFFFF
    sx = ((item >> 20) & 0xF) * 4
    sy = ((item >> 24) & 0x3) * 16
    code = (item >> 26) & 0x7
    rows = (code + 1) * (2 if chroma else 4)
    plane = (item >> 29) & 1
    return pu, sx, sy, rows, plane


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_mc_strips_cover_every_pu_once(hb, name):
    c = CONFIGS[name]
    pic = hb.Picture(hb.default_cfg(c["w"], c["h"], c["seed"], **c["cfg"]))
    s = pic.syn
    pus = [s.pus[i] for i in range(s.num_pus)]
    assert pus
    luma, chroma = hb.mc_strips(pic)
    for lst, is_chroma, planes in ((luma, False, 1), (chroma, True, 2)):
        cover = [[np.zeros(((u.h // (2 if is_chroma else 1)), (u.w // (2 if is_chroma else 1))), np.int32)
                  for _ in range(planes)] for u in pus]
        last_bi, last_rows, rises = 0, 1 << 30, 0
        for it in lst.tolist():
            pu, sx, sy, rows, plane = decode(it, is_chroma)
            u = pus[pu]
            cover[pu][plane][sy:sy + rows, sx:sx + 4] += 1
            bi = 0 if (u.ref_idx[0] >= 0 and u.ref_idx[1] >= 0) else 1
            assert bi >= last_bi, "bi-predicted strips first"
            last_bi = bi
            rises += rows > last_rows
            last_rows = rows
        # four classes (bi or not, windows inside the picture or not), taller strips first
        # in each: the row count only rises where a class starts
        assert rises <= 3, (name, is_chroma, rises)
        for k, u in enumerate(pus):
            for p in range(planes):
                assert np.all(cover[k][p] == 1), (name, is_chroma, k, p)
