"""The random-syntax bitstream generator (hevc.js_b200/bitgen.py, csrc/bitgen.cpp).

A generated stream is valid HEVC exactly when the reference decoder parses it into the syntax
the generator drew.  The reference's own decoder, run with the recorder inside it
(oracle/_ref/hevc-record: records every TU and PU it parses, and checks the oracle's
reconstruction of each picture against the reference's), gives the records; they must equal
the generator's, TU by TU and level by level, and PU by PU in position, size and (for a PU
coded with AMVP) reference indices; a merged PU's motion, and an AMVP PU's motion vector,
are the decoder's derivation, which the reconstruction check covers.  The drop-in decoder's host code (its parser
and recording hooks, over the CPU back end) and, on a GPU, the drop-in library must then give
the reference's frames."""
import ctypes as C
import hashlib
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(oracle.HERE, "_ref")
RECORDER = os.path.join(REF, "hevc-record")
REF_LIB = os.path.join(REF, "libhevcdec.so")

CONFIGS = {
    "64x64, defaults": dict(w=64, h=64, seed=1),
    "416x240, 16x16 CTBs, dense levels": dict(w=416, h=240, seed=2, log2_ctb=4, p_cbf=0.9, p_sig=0.8, max_level=4000),
    "200x136, 32x32 CTBs, all NxN": dict(w=200, h=136, seed=3, log2_ctb=5, p_split=0.8, p_nxn=1.0, qp_min=0, qp_max=12),
    "256x128, large blocks, no SAO": dict(w=256, h=128, seed=4, p_split=0.2, p_tu_split=0.0, sao=0, qp_min=45, qp_max=51),
    "72x40, three pictures": dict(w=72, h=40, seed=5, pictures=3, p_cbf=0.95),
    "P 64x64, one reference, no AMP or TMVP": dict(w=64, h=64, seed=11, inter=1, pictures=4, p_b=0.0, max_refs=1,
                                                   amp=0, tmvp=0),
    "B 64x64, AMP, TMVP": dict(w=64, h=64, seed=12, inter=1, pictures=4, p_b=1.0),
    "P/B 416x240, 32x32 CTBs, four references": dict(w=416, h=240, seed=13, inter=1, pictures=5, log2_ctb=5,
                                                     max_refs=4),
    "P/B 200x136, weighted prediction, far motion": dict(w=200, h=136, seed=14, inter=1, pictures=5, log2_ctb=4,
                                                         wp=1, max_mvd=4000),
    "P/B 72x40, interSplitFlag, one merge candidate": dict(w=72, h=40, seed=15, inter=1, pictures=6,
                                                           depth_inter=0, max_merge=1),
    "P/B 128x64, mostly skipped, dense residual": dict(w=128, h=64, seed=16, inter=1, pictures=5, p_skip=0.6,
                                                       p_cbf=0.9, p_sig=0.7, qp_min=0, qp_max=20),
}


def _needs_reference():
    if not (os.path.exists(RECORDER) and os.path.exists(REF_LIB)):
        pytest.skip("the reference decoder is not built (oracle/Makefile)")


def _generate(name):
    from hevc_b200 import bitgen
    c = dict(CONFIGS[name])
    return bitgen.generate(c.pop("w"), c.pop("h"), c.pop("seed"), **c)


def _md5(frames):
    return hashlib.md5(b"".join(f.yuv_bytes() for f in frames)).hexdigest()


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_reference_parses_the_drawn_syntax(hb, tmp_path, name):
    _needs_reference()
    from hevc_b200 import bitgen
    data, pics = _generate(name)
    stream, dump = tmp_path / "g.265", tmp_path / "g.hrec"
    stream.write_bytes(data)
    r = subprocess.run([RECORDER, str(stream), str(dump)], capture_output=True, text=True, timeout=120)
    summary = r.stdout.strip().split("\n")[-1]
    n = len(pics)
    assert summary == f"pictures {n} matched {n} mismatched 0 unsupported 0 decode_rc 0", r.stdout[-2000:] + r.stderr
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import real_streams
    rec = real_streams.load(hb.abi, str(dump))
    assert len(rec) == n
    key = lambda t: (t.c_idx, t.y, t.x)   # noqa: E731
    for k, (g, r_pic) in enumerate(zip(pics, rec)):
        levels = g.levels
        raw = r_pic.arrays["tus"].tobytes()
        got = sorted((hb.abi.TU.from_buffer_copy(raw, 16 * i) for i in range(len(raw) // 16)), key=key)
        want = sorted(g.tus, key=key)
        assert len(got) == len(want), (name, k)
        r_levels = r_pic.arrays["coeffs"]
        for a, b in zip(want, got):
            coded = a.flags & hb.abi.HEVC_TU_CODED
            fa = (a.x, a.y, a.log2_size, a.c_idx, a.intra_mode, a.flags, a.qp if coded else None)
            fb = (b.x, b.y, b.log2_size, b.c_idx, b.intra_mode, b.flags, b.qp if b.flags & hb.abi.HEVC_TU_CODED else None)
            assert fa == fb, (name, k)
            if coded:
                nn = 1 << (2 * a.log2_size)
                assert np.array_equal(levels[a.coeff_offset:a.coeff_offset + nn],
                                      r_levels[b.coeff_offset:b.coeff_offset + nn]), (name, k, fa)
        raw = r_pic.arrays["pus"].tobytes()
        size = C.sizeof(hb.abi.PU)
        pkey = lambda u: (u.y, u.x)   # noqa: E731
        got = sorted((hb.abi.PU.from_buffer_copy(raw, size * i) for i in range(len(raw) // size)), key=pkey)
        want = sorted(g.pus, key=pkey)
        assert [(u.x, u.y, u.w, u.h) for u in got] == [(u.x, u.y, u.w, u.h) for u in want], (name, k)
        for a, b in zip(want, got):
            if a.ref_idx[0] != -2:   # coded with AMVP: the lists used and the indices
                assert (a.ref_idx[0], a.ref_idx[1]) == (b.ref_idx[0], b.ref_idx[1]), (name, k, a.x, a.y)
        if g.slice_type == bitgen.SLICE_I:
            assert not want


def test_inter_streams_hold_every_kind_of_pu():
    """The inter configurations together draw every PU kind the syntax has: skipped and
    merged PUs, AMVP PUs of each direction, every partition shape."""
    from hevc_b200 import bitgen
    shapes, kinds = set(), set()
    for name, c in CONFIGS.items():
        if not c.get("inter"):
            continue
        _, pics = _generate(name)
        assert pics[0].slice_type == bitgen.SLICE_I
        assert all(p.slice_type in (bitgen.SLICE_P, bitgen.SLICE_B) for p in pics[1:])
        for p in pics:
            for u in p.pus:
                shapes.add((u.w, u.h))
                kinds.add("merge" if u.ref_idx[0] == -2 else
                          "bi" if min(u.ref_idx[0], u.ref_idx[1]) >= 0 else "l0" if u.ref_idx[0] >= 0 else "l1")
    assert kinds == {"merge", "l0", "l1", "bi"}
    ratios = {(w // min(w, h), h // min(w, h)) if w % h == 0 or h % w == 0 else (w, h) for w, h in shapes}
    assert {(1, 1), (2, 1), (1, 2), (4, 1), (1, 4)} <= ratios   # 2Nx2N, halves, AMP quarters
    assert any(w * 4 == h * 3 or h * 4 == w * 3 for w, h in shapes)   # AMP three quarters


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_dropin_host_code_decodes_generated_streams(name):
    """libhevcdec_oracle.so: the drop-in's parser and hooks over the CPU back end."""
    _needs_reference()
    from hevc_b200 import decoder as D
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    data, pics = _generate(name)
    ref = D.Decoder(REF_LIB)
    assert ref.decode(data) == 0
    want = ref.frames()
    assert len(want) == len(pics)
    dec = D.Decoder(checker)
    assert dec.decode(data) == 0, dec.last_error()
    assert _md5(dec.frames()) == _md5(want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_gpu_dropin_decodes_generated_streams(name):
    """libhevcdec_gpu.so on the generated streams: the reference's frames."""
    _needs_reference()
    from hevc_b200 import decoder as D
    data, pics = _generate(name)
    ref = D.Decoder(REF_LIB)
    assert ref.decode(data) == 0
    dec = D.Decoder()
    assert dec.decode(data) == 0, dec.last_error()
    assert _md5(dec.frames()) == _md5(ref.frames())
    assert dec.gpu_stats()[0] == len(pics)
