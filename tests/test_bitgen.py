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

# every test here imports the package (the generator, the decoder wrapper)
pytestmark = pytest.mark.usefixtures("hb")

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
    "I 200x136, cu_qp_delta, chroma QP offsets, deblocking control, slices": dict(
        w=200, h=136, seed=21, pictures=2, log2_ctb=5, qp_delta_depth=2, chroma_qp_offsets=1, deblock_ctl=1, slices=4),
    "P/B 208x120, cu_qp_delta, transform skip, sign hiding, 16x16 CTBs": dict(
        w=208, h=120, seed=22, inter=1, pictures=4, log2_ctb=4, qp_delta_depth=3, p_tskip=0.5, sdh=1),
    "P/B 200x136, scaling lists in the SPS, WPP": dict(w=200, h=136, seed=23, inter=1, pictures=4, log2_ctb=5,
                                                       scaling=2, wpp=1, chroma_qp_offsets=1),
    "P/B 416x240, slices, deblocking control, default scaling lists": dict(
        w=416, h=240, seed=26, inter=1, pictures=3, slices=5, deblock_ctl=1, scaling=1, qp_delta_depth=1),
    "I 128x64, scaling lists in the PPS, transquant bypass": dict(w=128, h=64, seed=24, pictures=2, scaling=3,
                                                                  p_bypass=0.3, p_tskip=0.3, sdh=1),
    "B 200x136, random access, mini-GOPs of 8, four references": dict(
        w=200, h=136, seed=31, inter=1, pictures=11, ra_gop=8, max_refs=4, p_b=1.0, log2_ctb=5),
    "P/B 208x120, random access, mini-GOPs of 4, weighted prediction": dict(
        w=208, h=120, seed=32, inter=1, pictures=10, ra_gop=4, wp=1, log2_ctb=4),
    "P/B 128x64, random access, mini-GOPs of 2, slices, cu_qp_delta": dict(
        w=128, h=64, seed=33, inter=1, pictures=7, ra_gop=2, slices=3, qp_delta_depth=2),
    "P/B 1920x1080, random access, mini-GOPs of 4, cu_qp_delta, deblocking control": dict(
        w=1920, h=1080, seed=4242, inter=1, pictures=8, ra_gop=4, p_b=0.8, max_refs=3, log2_ctb=6, p_cbf=0.3,
        p_sig=0.15, max_level=40, qp_min=22, qp_max=37, qp_delta_depth=2, deblock_ctl=1, p_skip=0.35, p_merge=0.5,
        p_intra_cu=0.05),
    "P/B 200x136, an IDR picture every 6, random access, cropping window": dict(
        w=200, h=136, seed=34, inter=1, pictures=14, ra_gop=4, idr_period=6, crop=1, log2_ctb=5),
    "I 120x72, cropping window": dict(w=120, h=72, seed=35, pictures=3, crop=1, log2_ctb=4),
    "P/B 200x136, list modification, long-term, slices, AUD/SEI/filler/EOS/VUI": dict(
        w=200, h=136, seed=38, inter=1, pictures=8, list_mod=1, long_term=1, slices=3, extra_syntax=1),
    "P/B 208x120, random access, list modification, an IDR picture every 4, AUD/SEI/VUI": dict(
        w=208, h=120, seed=39, inter=1, pictures=10, ra_gop=2, idr_period=4, list_mod=1, extra_syntax=1),
    "B 200x136, random access, mini-GOPs of 8, RPS sets in the SPS (inter RPS prediction)": dict(
        w=200, h=136, seed=40, inter=1, pictures=17, ra_gop=8, max_refs=3, sps_rps=1, p_b=1.0),
    "P/B 72x40, low delay, RPS sets in the SPS, long-term": dict(
        w=72, h=40, seed=41, inter=1, pictures=10, sps_rps=1, long_term=1, max_refs=3),
    "P/B 200x136, random access with CRA pictures (RASL and RADL leading pictures)": dict(
        w=200, h=136, seed=42, inter=1, pictures=17, ra_gop=4, cra=1, tmvp=1),
    "P/B 72x40, 40 pictures, POC LSBs of 4 bits (wrapping), long-term": dict(
        w=72, h=40, seed=43, inter=1, pictures=40, poc_lsb_bits=4, long_term=1, max_refs=3),
    "P/B 72x40, 40 pictures, random access with CRA pictures, POC LSBs of 4 bits": dict(
        w=72, h=40, seed=44, inter=1, pictures=40, poc_lsb_bits=4, ra_gop=4, cra=1),
    "P/B 200x136, an IDR picture every 4 with a new size (SPS and PPS sent again)": dict(
        w=200, h=136, seed=45, inter=1, pictures=16, idr_period=4, resize=1, crop=1),
    "I 200x136, a new size at every picture": dict(w=200, h=136, seed=46, pictures=6, resize=1),
    "B 200x136, random access, mini-GOPs of 8, temporal sub-layers, CRA pictures": dict(
        w=200, h=136, seed=47, inter=1, pictures=17, ra_gop=8, temporal=1, cra=1, p_b=1.0),
    "P/B 200x136, 40 pictures, CRA pictures, non-reference NAL types, POC LSBs of 4 bits": dict(
        w=200, h=136, seed=49, inter=1, pictures=40, ra_gop=4, cra=1, nonref_types=1, poc_lsb_bits=4),
    "P/B 200x136, four PPSs (cu_qp_delta, chroma offsets, deblocking, transform skip, WP, lists)": dict(
        w=200, h=136, seed=50, inter=1, pictures=8, pps_count=4, qp_delta_depth=2, chroma_qp_offsets=1,
        deblock_ctl=1, p_tskip=0.3, sdh=1, list_mod=1, wp=1),
    "P/B 200x136, long-term reference pictures, an IDR picture every 5": dict(
        w=200, h=136, seed=37, inter=1, pictures=12, long_term=1, idr_period=5, max_refs=2, tmvp=1),
    # written the way the reference reads these tools (HEVCGEN_QUIRK_*): see
    # test_reference_reads_these_tools_its_own_way
    "I 640x256, 2x3 tiles, slices [reference's tile reading]": dict(
        w=640, h=256, seed=25, pictures=2, log2_ctb=5, tile_cols=2, tile_rows=3, slices=4, ref_quirks=1),
    "P/B 528x256, 2x2 tiles, cu_qp_delta [reference's tile reading]": dict(
        w=528, h=256, seed=27, inter=1, pictures=3, log2_ctb=4, tile_cols=2, tile_rows=2, qp_delta_depth=2,
        ref_quirks=1),
    "I 200x136, PCM, cu_qp_delta [reference's PCM reading]": dict(w=200, h=136, seed=28, pictures=2, log2_ctb=5,
                                                                  p_pcm=0.3, qp_delta_depth=2, ref_quirks=1),
    "P/B 200x136, dependent slice segments [reference's reading]": dict(
        w=200, h=136, seed=29, inter=1, pictures=3, log2_ctb=6, slices=5, dependent_slices=1, ref_quirks=2),
}

# pictures the recorder cannot replay (the oracle sees no levels for PCM and bypass CUs):
# their records are still compared, with the replay check skipped
UNREPLAYED = {name for name, c in CONFIGS.items() if c.get("p_pcm") or c.get("p_bypass")}


def _needs_reference():
    if not (os.path.exists(RECORDER) and os.path.exists(REF_LIB)):
        pytest.skip("the reference decoder is not built (oracle/Makefile)")


def _generate(name):
    from hevc_b200 import bitgen
    c = dict(CONFIGS[name])
    return bitgen.generate(c.pop("w"), c.pop("h"), c.pop("seed"), **c)


def _as_parsed(abi, tus):
    """The generator's TU records as the recorder sees the reference parse them: no record
    for PCM blocks or for the blocks of an inter bypass CU, and the blocks of an intra bypass
    CU as intra blocks without levels (the reference dequantises neither)."""
    out = []
    for t in tus:
        if t.flags & abi.HEVC_TU_PCM or (t.flags & abi.HEVC_TU_BYPASS and not t.flags & abi.HEVC_TU_INTRA):
            continue
        if t.flags & abi.HEVC_TU_BYPASS:
            t = abi.TU.from_buffer_copy(t)
            t.flags = abi.HEVC_TU_INTRA
        out.append(t)
    return out


def _output_order(pics):
    """POCs in output order: period by period (an IDR picture starts one), each in POC order."""
    out, period = [], []
    for g in pics:
        if g.slice_type == 2 and g.poc == 0 and period:
            out += sorted(period)
            period = []
        period.append(g.poc)
    return out + sorted(period)


def _md5(frames):
    return hashlib.md5(b"".join(f.yuv_bytes() for f in frames)).hexdigest()


def _record(tmp_path, data):
    """The reference's recorder on a stream: its summary line and the records of every
    picture up to the first mismatched one."""
    stream, dump = tmp_path / "g.265", tmp_path / "g.hrec"
    stream.write_bytes(data)
    r = subprocess.run([RECORDER, str(stream), str(dump), "--all"], capture_output=True, text=True, timeout=120)
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import real_streams
    return r.stdout.strip().split("\n")[-1], real_streams.load(_abi(), str(dump)), r.stdout[-2000:] + r.stderr


def _abi():
    from hevc_b200 import abi
    return abi


def _differences(pics, rec):
    """Where the records the reference parsed differ from the drawn ones: TUs (position,
    size, plane, mode, flags, QP and levels of coded ones), PUs (position and size; an
    AMVP-coded PU's reference indices).  Empty when the reference parsed what was drawn."""
    abi = _abi()
    out = []
    if len(rec) != len(pics):
        out.append(("pictures recorded", len(rec), len(pics)))
    key = lambda t: (t.c_idx, t.y, t.x)   # noqa: E731
    for k, (g, r_pic) in enumerate(zip(pics, rec)):
        raw = r_pic.arrays["tus"].tobytes()
        got = sorted((abi.TU.from_buffer_copy(raw, 16 * i) for i in range(len(raw) // 16)), key=key)
        want = sorted(_as_parsed(abi, g.tus), key=key)
        if len(got) != len(want):
            out.append((k, "TU count", len(want), len(got)))
            continue
        r_levels = r_pic.arrays["coeffs"]
        for a, b in zip(want, got):
            coded = a.flags & abi.HEVC_TU_CODED
            fa = (a.x, a.y, a.log2_size, a.c_idx, a.intra_mode, a.flags, a.qp if coded else None)
            fb = (b.x, b.y, b.log2_size, b.c_idx, b.intra_mode, b.flags, b.qp if b.flags & abi.HEVC_TU_CODED else None)
            nn = 1 << (2 * a.log2_size)
            if fa != fb or (coded and not np.array_equal(g.levels[a.coeff_offset:a.coeff_offset + nn],
                                                         r_levels[b.coeff_offset:b.coeff_offset + nn])):
                out.append((k, "TU", fa, fb))
                break
        raw = r_pic.arrays["pus"].tobytes()
        size = C.sizeof(abi.PU)
        pkey = lambda u: (u.y, u.x)   # noqa: E731
        got = sorted((abi.PU.from_buffer_copy(raw, size * i) for i in range(len(raw) // size)), key=pkey)
        want = sorted(g.pus, key=pkey)
        if [(u.x, u.y, u.w, u.h) for u in got] != [(u.x, u.y, u.w, u.h) for u in want]:
            out.append((k, "PU layout"))
            continue
        for a, b in zip(want, got):
            if a.ref_idx[0] != -2 and (a.ref_idx[0], a.ref_idx[1]) != (b.ref_idx[0], b.ref_idx[1]):
                out.append((k, "PU reference indices", a.x, a.y))
                break
    return out


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_reference_parses_the_drawn_syntax(hb, tmp_path, name):
    _needs_reference()
    from hevc_b200 import bitgen
    data, pics = _generate(name)
    summary, rec, log = _record(tmp_path, data)
    n = len(pics)
    if name in UNREPLAYED:   # intra pictures only: the replay is skipped, the records are written
        f = summary.split()
        assert f[0] == "pictures" and int(f[1]) == n and f[5] == "0" and f[9] == "0", log
        assert int(f[3]) + int(f[7]) == n and int(f[7]) >= 1, summary
    else:
        assert summary == f"pictures {n} matched {n} mismatched 0 unsupported 0 decode_rc 0", log
    assert _differences(pics, rec) == []
    for g in pics:
        if g.slice_type == bitgen.SLICE_I:
            assert not g.pus


TEN_BIT = [name for name in sorted(CONFIGS) if any(k in name for k in (
    "chroma QP offsets", "PCM", "weighted prediction", "scaling lists in the SPS", "2x2 tiles",
    "dependent slice segments", "sign hiding", "dense levels"))]


@pytest.mark.parametrize("name", TEN_BIT)
def test_reference_parses_the_drawn_syntax_at_10_bits(tmp_path, name):
    """Main10 streams (BitDepthY = BitDepthC = 10): the reference parses every picture into
    the drawn records.  Their QP is Qp' (QpY + QpBdOffset, 8.6.1), SAO offsets reach 31
    (7.4.9.3.2), PCM samples up to 10 bits.  The oracle and the kernels keep 8-bit
    samples, so the recorder marks the pictures unsupported and only the records are
    compared."""
    _needs_reference()
    from hevc_b200 import bitgen
    c = dict(CONFIGS[name], bit_depth=10)
    data, pics = bitgen.generate(c.pop("w"), c.pop("h"), c.pop("seed"), **c)
    summary, rec, log = _record(tmp_path, data)
    n = len(pics)
    assert summary == f"pictures {n} matched 0 mismatched 0 unsupported {n} decode_rc 0", log
    assert _differences(pics, rec) == []
    # luma Qp' = QpY + 12 (QpY >= 0 here); the parsed records carry the same
    assert all(t.qp >= 12 for g in pics for t in g.tus if t.c_idx == 0)


def test_dropin_refuses_10_bit_streams():
    """The drop-in keeps 8-bit samples: a Main10 stream fails at its first picture with a
    message, and no frame is handed out."""
    _needs_reference()
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    from hevc_b200 import bitgen, decoder as D
    data, _ = bitgen.generate(64, 64, 1, bit_depth=10)
    dec = D.Decoder(checker)
    assert dec.decode(data) != 0
    assert "bit" in dec.last_error()
    assert dec.frames() == []


def test_generator_bit_depths():
    from hevc_b200 import bitgen
    a, _ = bitgen.generate(64, 64, 1)
    b, _ = bitgen.generate(64, 64, 1, bit_depth=8)
    assert a == b
    with pytest.raises(Exception):
        bitgen.generate(64, 64, 1, bit_depth=9)


# Where the reference's parser departs from H.265 (each found with these streams): a stream
# written by the standard is not parsed into what was drawn, the same stream written the
# way the reference reads it is.  Details at the HEVCGEN_QUIRK_* bits (csrc/bitgen.h).
DEPARTURES = {
    "tiles: contexts at a tile start, alignment after end_of_subset_one_bit": (
        dict(w=832, h=256, seed=1, pictures=3, log2_ctb=5, tile_cols=3, tile_rows=3), 1),
    "PCM: alignment after pcm_flag, contexts after the samples": (
        dict(w=200, h=136, seed=1, pictures=1, log2_ctb=5, p_pcm=0.3), 1),
    "dependent slice segments: availability per segment, header alignment": (
        dict(w=200, h=136, seed=2, pictures=1, log2_ctb=6, slices=4, dependent_slices=1), 2),
}


@pytest.mark.parametrize("name", sorted(DEPARTURES))
def test_reference_reads_these_tools_its_own_way(tmp_path, name):
    _needs_reference()
    from hevc_b200 import bitgen
    cfg, quirk = DEPARTURES[name]
    c = dict(cfg)
    w, h, seed = c.pop("w"), c.pop("h"), c.pop("seed")
    data, pics = bitgen.generate(w, h, seed, **c)
    _, rec, _ = _record(tmp_path, data)
    assert _differences(pics, rec), "the reference now parses the standard's form"
    data, pics = bitgen.generate(w, h, seed, ref_quirks=quirk, **c)
    _, rec, log = _record(tmp_path, data)
    assert _differences(pics, rec) == [], log


def test_reference_outputs_pictures_whose_pic_output_flag_is_0():
    """Another departure, in the output process: pic_output_flag = 0 makes PicOutputFlag 0
    (8.1.3), so the picture is never output (C.5.2); the reference marks every picture as
    needed for output (decoder.cpp:298, after :85 had taken the flag).  Reading its code, it
    does not apply no_output_of_prior_pics_flag either (parsed at slice_header.cpp:124 and not
    used), which C.5.2.2 applies at an IDR picture."""
    _needs_reference()
    from hevc_b200 import bitgen, decoder as D
    data, pics = bitgen.generate(200, 136, 36, inter=1, pictures=8, ra_gop=4, p_no_output=0.5)
    assert not all(g.output for g in pics)
    ref = D.Decoder(REF_LIB)
    assert ref.decode(data) == 0
    assert [f.poc for f in ref.frames()] == _output_order(pics)   # every picture, the hidden ones too


def test_generated_cropping_windows():
    """A cropping window is drawn: the reference's frames have the cropped size."""
    _needs_reference()
    from hevc_b200 import bitgen, decoder as D
    data, pics = _generate("I 120x72, cropping window")
    ref = D.Decoder(REF_LIB)
    assert ref.decode(data) == 0
    f = ref.frames()[0]
    assert (f.width, f.height) != (120, 72) and f.width >= 16 and f.height >= 16


def _from_a_cra(seed):
    """A random-access stream with CRA pictures, cut at its first CRA picture (the parameter
    sets kept), and the POCs of that picture's RASL pictures."""
    from hevc_b200 import bitgen
    data, pics = bitgen.generate(200, 136, seed, inter=1, pictures=17, ra_gop=4, cra=1)
    pos = [k for k in range(len(data) - 3) if data[k:k + 4] == b"\x00\x00\x00\x01"]
    nals = [data[a:b] for a, b in zip(pos, pos[1:] + [len(data)])]
    types = [(n[4] >> 1) & 63 for n in nals]
    vcl = [t for t in types if t < 32]   # one slice per picture: one VCL NAL unit each
    assert 21 in vcl, "no CRA picture drawn"
    first, k = vcl.index(21), types.index(21)
    cut = b"".join([n for n, t in zip(nals, types) if t in (32, 33, 34)] + nals[k:])
    rasl = {pics[i].poc for i in range(first + 1, len(pics)) if vcl[i] in (8, 9) and pics[i].poc < pics[first].poc}
    return cut, rasl


def _check_from_a_cra(lib, seed):
    from hevc_b200 import decoder as D
    cut, rasl = _from_a_cra(seed)
    assert rasl
    ref = D.Decoder(REF_LIB)
    assert ref.decode(cut) == 0
    want = ref.frames()
    runs = []
    for _ in range(2):
        dec = D.Decoder(lib)
        assert dec.decode(cut) == 0, dec.last_error()
        runs.append(dec.frames())
    got = runs[0]
    assert [f.poc for f in got] == [f.poc for f in want]
    for f, g in zip(got, want):
        if f.poc not in rasl:
            assert _md5([f]) == _md5([g]), f.poc
    assert _md5(runs[0]) == _md5(runs[1])   # the RASL pictures too: deterministic


@pytest.mark.parametrize("seed", [1, 3])
def test_decoding_from_a_cra_picture(seed):
    """Random access at a CRA picture: its RASL pictures have references the decoder never
    saw.  The drop-in predicts from the generated picture of 8.3.3.2 there (the reference
    reads an uninitialised buffer, interpolation.cpp:327-331, and the standard outputs no
    such picture); every other picture is the reference's, in the reference's output order."""
    _needs_reference()
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    _check_from_a_cra(checker, seed)


@pytest.mark.gpu
@pytest.mark.last
@pytest.mark.parametrize("seed", [1, 3])
def test_gpu_decoding_from_a_cra_picture(seed):
    _needs_reference()
    _check_from_a_cra(None, seed)


def _with_a_slice_twice():
    """A generated stream in which the second slice of the first picture is sent again after
    the picture's last one: those CTUs are coded twice (a damaged stream)."""
    from hevc_b200 import bitgen
    data, _ = bitgen.generate(200, 136, 7, inter=1, pictures=3, slices=4, log2_ctb=4)
    pos = [k for k in range(len(data) - 3) if data[k:k + 4] == b"\x00\x00\x00\x01"]
    nals = [data[a:b] for a, b in zip(pos, pos[1:] + [len(data)])]
    vcl = [i for i, n in enumerate(nals) if ((n[4] >> 1) & 63) < 32]
    starts = [i for i in vcl if nals[i][6] & 0x80]   # first_slice_segment_in_pic_flag
    pic0 = [i for i in vcl if starts[0] <= i < starts[1]]
    assert len(pic0) >= 2
    return b"".join(nals[:pic0[-1] + 1] + [nals[pic0[1]]] + nals[pic0[-1] + 1:])


def _check_slice_twice(lib):
    from hevc_b200 import decoder as D
    data = _with_a_slice_twice()
    ref = D.Decoder(REF_LIB)
    assert ref.decode(data) == 0   # the reference keeps whichever coding came last
    dec = D.Decoder(lib)
    assert dec.decode(data) != 0
    assert "code some blocks more than once" in dec.last_error()


def test_a_picture_whose_slices_overlap_fails():
    """The drop-in refuses a picture whose slices code some blocks twice, with a message,
    where its records cannot say which coding the reference kept."""
    _needs_reference()
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    _check_slice_twice(checker)


@pytest.mark.gpu
@pytest.mark.last
def test_gpu_a_picture_whose_slices_overlap_fails():
    _needs_reference()
    _check_slice_twice(None)


def _with_a_slice_header_cut():
    """A generated stream cut two bytes into the header of the last picture's second slice."""
    from hevc_b200 import bitgen
    data, _ = bitgen.generate(200, 136, 7, inter=1, pictures=3, slices=4, log2_ctb=4)
    pos = [k for k in range(len(data) - 3) if data[k:k + 4] == b"\x00\x00\x00\x01"]
    nals = [data[a:b] for a, b in zip(pos, pos[1:] + [len(data)])]
    vcl = [i for i, n in enumerate(nals) if ((n[4] >> 1) & 63) < 32]
    starts = [i for i in vcl if nals[i][6] & 0x80]   # first_slice_segment_in_pic_flag
    last = [i for i in vcl if i >= starts[-1]]
    assert len(starts) == 3 and len(last) >= 2
    return b"".join(nals[:last[1]]) + nals[last[1]][:8]


def _check_slice_header_cut(lib):
    from hevc_b200 import decoder as D
    data = _with_a_slice_header_cut()
    ref = D.Decoder(REF_LIB)
    assert ref.decode(data) == 0
    want = ref.frames()
    assert [f.poc for f in want] == [0, 1, 2]   # POC 2's slices were never decoded
    dec = D.Decoder(lib)
    assert dec.decode(data) == 0, dec.last_error()
    got = dec.frames()
    assert [f.poc for f in got] == [0, 1]
    assert _md5(got) == _md5(want[:2])


def test_a_picture_cut_short_is_not_handed_out():
    """A picture whose second slice header fails to parse: the reference still outputs it
    (decoder.cpp:85 marks it for output when it is allocated; decoder.cpp:198-201 returns
    before any of its slice data is decoded), with whatever samples its reused buffer held.
    The drop-in hands out no frame for a picture it did not reconstruct, and every other
    frame is the reference's."""
    _needs_reference()
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    _check_slice_header_cut(checker)


@pytest.mark.gpu
@pytest.mark.last
def test_gpu_a_picture_cut_short_is_not_handed_out():
    _needs_reference()
    _check_slice_header_cut(None)


def _without_a_current_reference():
    """A generated P picture whose RPS marks its one reference as not used by it
    (used_by_curr_pic_s0_flag flipped): NumPicTotalCurr is 0, which 7.4.7.2 forbids in a P
    slice (a damaged stream)."""
    from hevc_b200 import bitgen
    data, _ = bitgen.generate(64, 64, 5, inter=1, pictures=3, max_refs=1, p_b=0.0, sao=0, tmvp=0)
    pos = [k for k in range(len(data) - 3) if data[k:k + 4] == b"\x00\x00\x00\x01"]
    nals = [data[a:b] for a, b in zip(pos, pos[1:] + [len(data)])]
    k = [(n[4] >> 1) & 63 for n in nals].index(1)   # the first P picture (TRAIL_R)
    n = bytearray(nals[k])
    bits = "".join(f"{b:08b}" for b in n[6:10])
    # first_slice_segment_in_pic_flag, pps id, slice_type P, 8 POC LSBs, sps flag 0,
    # num_negative_pics 1, num_positive_pics 0, delta_poc_s0_minus1 0, then the flag
    assert bits[:5] == "11010" and bits[13:17] == "0010" and bits[17:19] == "11", bits
    n[6 + 19 // 8] ^= 0x80 >> (19 % 8)
    nals[k] = bytes(n)
    return b"".join(nals)


def _check_without_a_current_reference(lib):
    from hevc_b200 import decoder as D
    dec = D.Decoder(lib)
    assert dec.decode(_without_a_current_reference()) != 0
    assert "without a current reference picture" in dec.last_error()


def test_a_slice_without_a_current_reference_fails(tmp_path):
    """The drop-in refuses a P/B slice with NumPicTotalCurr 0; the reference's list
    construction does not end on it (dpb.cpp:259-266: checked in a child process with a
    time limit)."""
    _needs_reference()
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    _check_without_a_current_reference(checker)
    stream = tmp_path / "nocurr.265"
    stream.write_bytes(_without_a_current_reference())
    code = ("import sys; sys.path.insert(0, %r); import __graft_entry__ as ge; ge.load_package(); "
            "from hevc_b200 import decoder as D; D.Decoder(%r).decode(open(%r, 'rb').read())"
            % (os.path.dirname(HERE), REF_LIB, str(stream)))
    with pytest.raises(subprocess.TimeoutExpired):
        subprocess.run([sys.executable, "-c", code], capture_output=True, timeout=5)


@pytest.mark.gpu
@pytest.mark.last
def test_gpu_a_slice_without_a_current_reference_fails():
    _check_without_a_current_reference(None)


def _check_sub_layers(lib):
    """Every temporal sub-bitstream (the NAL units of TemporalId <= T) decodes to the
    reference's frames: the pictures of those sub-layers, in POC order."""
    from hevc_b200 import bitgen, decoder as D
    data, pics = bitgen.generate(200, 136, 48, inter=1, pictures=17, ra_gop=8, temporal=1)
    pos = [k for k in range(len(data) - 3) if data[k:k + 4] == b"\x00\x00\x00\x01"]
    nals = [data[a:b] for a, b in zip(pos, pos[1:] + [len(data)])]
    top = max(g.tid for g in pics)
    assert top == 3
    for t in range(top + 1):
        sub = b"".join(n for n in nals if (n[5] & 7) - 1 <= t)   # nuh_temporal_id_plus1
        ref = D.Decoder(REF_LIB)
        assert ref.decode(sub) == 0
        want = ref.frames()
        assert [f.poc for f in want] == sorted(g.poc for g in pics if g.tid <= t)
        dec = D.Decoder(lib)
        assert dec.decode(sub) == 0, dec.last_error()
        assert _md5(dec.frames()) == _md5(want), t


def test_temporal_sub_bitstreams():
    _needs_reference()
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    _check_sub_layers(checker)


@pytest.mark.gpu
@pytest.mark.last
def test_gpu_temporal_sub_bitstreams():
    _needs_reference()
    _check_sub_layers(None)


def _one_ctu_wide(**kw):
    """A WPP stream of pictures one CTU wide (64x256, 64x64 CTUs): four CTU rows, each its own
    substream."""
    from hevc_b200 import bitgen
    return bitgen.generate(64, 256, 3, log2_ctb=6, wpp=1, **kw)


def _check_records_and_frames(port, tmp_path, lib, data, pics):
    """Where the unmodified reference cannot be the judge: the recorder (the reference's
    parser, on its sequential WPP path) must parse the drawn records and its oracle replay
    match, and the drop-in's frames must be the oracle's reconstruction of those records,
    in output order."""
    from hevc_b200 import decoder as D
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import real_streams
    summary, rec, log = _record(tmp_path, data)
    n = len(pics)
    assert summary == f"pictures {n} matched {n} mismatched 0 unsupported 0 decode_rc 0", log
    assert _differences(pics, rec) == []
    outs = real_streams.replay(port.reconstruct_picture, rec)   # decode order, packed I420
    want, period = [], []   # output order: period by period (an IDR picture starts one), by POC
    for g, o in zip(pics, outs):
        if g.slice_type == 2 and g.poc == 0 and period:
            want += sorted(period, key=lambda e: e[0])
            period = []
        period.append((g.poc, o))
    want += sorted(period, key=lambda e: e[0])
    dec = D.Decoder(lib)
    assert dec.decode(data) == 0, dec.last_error()
    frames = dec.frames()
    assert [f.poc for f in frames] == [e[0] for e in want]
    for f, (poc, w) in zip(frames, want):
        got = np.concatenate([pl.astype(np.uint8).ravel() for pl in f.planes])
        assert np.array_equal(got, w), poc
    return frames


def _wpp_slices(**kw):
    """A WPP stream of several slices per picture (some starting inside a CTU row)."""
    from hevc_b200 import bitgen
    return bitgen.generate(200, 136, 20, log2_ctb=5, wpp=1, slices=6, **kw)


def test_wpp_pictures_of_several_slices(port, tmp_path):
    """The reference's threaded WPP path decodes every row of a slice from column 0 to the
    picture's last row (coding_tree.cpp:404-533), so a picture of several slices is decoded
    from the wrong substreams.  The drop-in (and the recorder) give such pictures the
    reference's sequential path, which follows 9.3.1: the drawn records, and the oracle's
    reconstruction of them.  The unmodified reference's frames differ here (in 29 of 40
    such streams drawn: where its stray rows are not all coded again by a later slice)."""
    _needs_reference()
    from hevc_b200 import decoder as D
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    for kw in (dict(pictures=3), dict(inter=1, pictures=6, ra_gop=4, qp_delta_depth=2)):
        data, pics = _wpp_slices(**kw)
        frames = _check_records_and_frames(port, tmp_path, checker, data, pics)
        ref = D.Decoder(REF_LIB)
        assert ref.decode(data) == 0
        assert _md5(ref.frames()) != _md5(frames)


@pytest.mark.gpu
@pytest.mark.last
def test_gpu_wpp_pictures_of_several_slices():
    from hevc_b200 import decoder as D
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    for kw in (dict(pictures=3), dict(inter=1, pictures=6, ra_gop=4, qp_delta_depth=2)):
        data, _ = _wpp_slices(**kw)
        ref = D.Decoder(checker)
        assert ref.decode(data) == 0
        dec = D.Decoder()
        assert dec.decode(data) == 0, dec.last_error()
        assert _md5(dec.frames()) == _md5(ref.frames())


def test_wpp_pictures_one_ctu_wide(port, tmp_path):
    """The reference's threaded WPP path starts each CTU row once the row above has finished
    its second CTU (coding_tree.cpp:404-533); a picture one CTU wide has none, and the
    unmodified reference does not return (checked in a child process with a time limit).
    The drop-in (and the recorder) give such pictures the reference's sequential path: the
    reference then parses the drawn records, and the drop-in's frames are the oracle's
    reconstruction of them."""
    _needs_reference()
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    for kw in (dict(pictures=3), dict(inter=1, pictures=6, ra_gop=4)):
        _check_records_and_frames(port, tmp_path, checker, *_one_ctu_wide(**kw))
    stream = tmp_path / "wide1.265"
    stream.write_bytes(_one_ctu_wide(pictures=2)[0])
    code = ("import sys; sys.path.insert(0, %r); import __graft_entry__ as ge; ge.load_package(); "
            "from hevc_b200 import decoder as D; D.Decoder(%r).decode(open(%r, 'rb').read())"
            % (os.path.dirname(HERE), REF_LIB, str(stream)))
    with pytest.raises(subprocess.TimeoutExpired):
        subprocess.run([sys.executable, "-c", code], capture_output=True, timeout=5)


@pytest.mark.gpu
@pytest.mark.last
def test_gpu_wpp_pictures_one_ctu_wide():
    """The GPU drop-in on the same streams: the CPU checker's frames (the same host code over
    the oracle)."""
    from hevc_b200 import decoder as D
    checker = os.path.join(REF, "libhevcdec_oracle.so")
    if not os.path.exists(checker):
        pytest.skip("the drop-in checker is not built (oracle/Makefile)")
    for kw in (dict(pictures=3), dict(inter=1, pictures=6, ra_gop=4)):
        data, _ = _one_ctu_wide(**kw)
        ref = D.Decoder(checker)
        assert ref.decode(data) == 0
        dec = D.Decoder()
        assert dec.decode(data) == 0, dec.last_error()
        assert _md5(dec.frames()) == _md5(ref.frames())


def test_random_access_streams_are_reordered():
    """A random-access stream codes each mini-GOP's last picture first and the others by
    bisection; every POC appears once."""
    for name, c in CONFIGS.items():
        if c.get("ra_gop", 0) < 2:
            continue
        _, pics = _generate(name)
        pocs = [g.poc for g in pics]
        period = c.get("idr_period") or len(pics)
        assert sorted(pocs[:period]) == list(range(min(period, len(pics))))
        assert pocs != sorted(pocs), name
        assert pocs[1] == min(c["ra_gop"], period - 1)


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
        if not c.get("cra"):   # I slices in IDR pictures only (CRA pictures are I too)
            assert all((p.slice_type == bitgen.SLICE_I) == (p.poc == 0) for p in pics)
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
    got = dec.frames()
    assert _md5(got) == _md5(want)
    assert [f.poc for f in got] == [f.poc for f in want] == _output_order(pics)
    c = CONFIGS[name]
    for f, g in zip(got, want):   # the conformance window, the size of each picture
        assert (f.width, f.height) == (g.width, g.height)
        if not c.get("crop") and not c.get("resize"):
            assert (f.width, f.height) == (c["w"], c["h"])


@pytest.mark.gpu
@pytest.mark.last
@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_gpu_dropin_decodes_generated_streams(name):
    """libhevcdec_gpu.so on the generated streams: the reference's frames.  Run last: the
    widest spread of syntax through the GPU decoder."""
    _needs_reference()
    from hevc_b200 import decoder as D
    data, pics = _generate(name)
    ref = D.Decoder(REF_LIB)
    assert ref.decode(data) == 0
    dec = D.Decoder()
    assert dec.decode(data) == 0, dec.last_error()
    got = dec.frames()
    assert _md5(got) == _md5(ref.frames())
    assert [f.poc for f in got] == _output_order(pics)
    assert dec.gpu_stats()[0] == len(pics)
