"""The drop-in decoder: privaloops/hevc.js's own C API (src/wasm/hevc_api.h) over its own
host parser, with every picture reconstructed by the GPU back end.

The reference's conformance and demo streams (tests/golden/streams/) must decode to the
MD5s the reference's own decoder gives (tests/golden/streams.json, made by
tests/golden/make_streams_golden.py; for 11 of the 13 8-bit streams that is also the MD5 the
reference's test suite expects, CMakeLists.txt:139-224):

  - the whole output file, as the reference's CLI writes it, and every frame in the order
    hevc_decoder_get_frame hands them out;
  - every frame through hevc_decoder_feed per access unit with drain/flush, in bumping
    order (the property of the reference's tests/unit/test_incremental.cpp:50-176);
  - the reference's own CLI (src/main.cpp) linked against the drop-in library.

On the CPU the same host logic runs in a checker build (oracle/_ref/libhevcdec_oracle.so,
test infrastructure) whose pictures the oracle reconstructs; the GPU tests run the product
library, libhevcdec_gpu.so, and check that the GPU reconstructed every picture.
"""
import hashlib
import json
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
STREAMS = os.path.join(HERE, "golden", "streams")
with open(os.path.join(HERE, "golden", "streams.json")) as _f:
    GOLDEN = json.load(_f)
EIGHT_BIT = sorted(n for n, g in GOLDEN.items() if g["bit_depth"] == 8)
TEN_BIT = sorted(n for n, g in GOLDEN.items() if g["bit_depth"] != 8)


def _data(name):
    with open(os.path.join(STREAMS, name), "rb") as f:
        return f.read()


def _decode_batch(D, lib, name):
    dec = D.Decoder(lib)
    rc = dec.decode(_data(name))
    assert rc == 0, f"{name}: hevc_decoder_decode {rc}: {dec.last_error()}"
    frames = dec.frames()
    stats = dec.gpu_stats() if hasattr(dec.lib, "hevc_decoder_gpu_stats") else None
    dec.close()
    return frames, stats


def _decode_incremental(D, lib, name):
    dec = D.Decoder(lib)
    frames = []
    for chunk in D.split_access_units(_data(name)):
        assert dec.feed(chunk) == 0, f"{name}: hevc_decoder_feed: {dec.last_error()}"
        frames += dec.drain()
    frames += dec.flush()
    dec.close()
    return frames


def _check(name, frames, key="frames"):
    want = GOLDEN[name]
    got = [[f.poc, f.md5()] for f in frames]
    bad = [i for i, (a, b) in enumerate(zip(got, want[key])) if a != b]
    assert len(got) == len(want[key]) and not bad, f"{name}: {len(got)} frames, first differing {bad[:8]}"
    if key == "frames":
        whole = hashlib.md5(b"".join(f.yuv_bytes() for f in frames)).hexdigest()
        assert whole == want["md5"]
        if want["published"]:
            assert whole == want["published"]


@pytest.fixture(scope="module")
def D(hb):
    from hevc_b200 import decoder
    return decoder


@pytest.fixture(scope="module")
def checker_lib():
    import oracle
    if not os.path.exists(oracle.DROPIN_SO):
        if not os.path.isdir(os.path.join(oracle.REF_DIR, "src")):
            pytest.skip("the checker build needs the reference's parser sources")
        oracle.build()
    return oracle.DROPIN_SO


@pytest.fixture(scope="module")
def gpu_lib(hb):
    from hevc_b200 import build
    if not os.path.exists(build.DROPIN_SO):
        build.build_gpu()
        assert build.build_dropin(), "libhevcdec_gpu.so is built from the reference's parser sources"
    return build.DROPIN_SO


# ---- CPU: the library, the golden vectors, the host logic --------------------------------

def test_split_access_units_keeps_pictures_whole(D):
    data = _data("b_qcif_10f.265")
    chunks = D.split_access_units(data)
    assert b"".join(chunks) == data
    assert len(chunks) == len(GOLDEN["b_qcif_10f.265"]["frames"])


def test_golden_pins_the_published_md5s():
    published = [n for n, g in GOLDEN.items() if g["published"]]
    assert len(published) == 13   # every oracle test of the reference but the absent 4K stream
    for n in published:
        assert GOLDEN[n]["md5"] == GOLDEN[n]["published"]
        assert sorted(p for p, _ in GOLDEN[n]["incremental"]) == sorted(p for p, _ in GOLDEN[n]["frames"])


def test_dropin_library_exports_the_reference_api(gpu_lib):
    syms = subprocess.run(["nm", "-D", "--defined-only", gpu_lib], capture_output=True, text=True).stdout
    with open(os.path.join(os.path.dirname(HERE), "include", "hevc_api_gpu.h")) as f:
        header = f.read()
    import re
    declared = set(re.findall(r"\b(hevc_decoder_\w+)\s*\(", header))
    assert len(declared) == 14
    for name in declared:
        assert f" T {name}\n" in syms, name
    # the reconstruction hooks are this library's own recording definitions: the reference
    # objects that define them (and their CPU arithmetic) are not linked
    nm = subprocess.run(["nm", "-C", "--defined-only", gpu_lib], capture_output=True, text=True).stdout
    for hook in ("hevc::perform_dequant(", "hevc::perform_transform_inverse(", "hevc::perform_intra_prediction(",
                 "hevc::perform_inter_prediction(", "hevc::apply_deblocking(", "hevc::apply_sao("):
        assert nm.count(" T " + hook) == 1, hook
    for ref_only in ("interpolate_luma", "weighted_pred_explicit", "idct32", "filter_luma_sample", "band_offset"):
        assert ref_only not in nm, ref_only


def test_dropin_without_a_gpu_fails_loudly(D, gpu_lib):
    """No CPU fallback: with no CUDA device the first picture fails and nothing is handed out."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    dec = D.Decoder(gpu_lib)
    assert dec.decode(_data("toy_qp30.265")) == -1
    assert "GPU" in dec.last_error() or "CUDA" in dec.last_error()
    assert dec.frames() == []
    dec.close()


@pytest.mark.parametrize("name", EIGHT_BIT)
def test_checker_build_reproduces_reference_streams(D, checker_lib, name):
    frames, stats = _decode_batch(D, checker_lib, name)
    _check(name, frames)
    assert stats[0] == len(frames)


@pytest.mark.parametrize("name", ["full_qcif_10f.265", "b_qcif_10f.265", "p_qcif_10f.265", "bbb1080_singleslice.265"])
def test_checker_build_incremental_matches_batch(D, checker_lib, name):
    _check(name, _decode_incremental(D, checker_lib, name), "incremental")


@pytest.mark.parametrize("name", TEN_BIT)
def test_checker_build_refuses_ten_bit(D, checker_lib, name):
    dec = D.Decoder(checker_lib)
    assert dec.decode(_data(name)) == -1
    assert "bit depth 10" in dec.last_error()
    dec.close()


# ---- GPU: the product library ------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("name", EIGHT_BIT)
def test_gpu_dropin_reproduces_reference_streams(D, gpu_lib, name):
    frames, (pictures, launches) = _decode_batch(D, gpu_lib, name)
    _check(name, frames)
    assert pictures == len(frames) and launches >= pictures


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["full_qcif_10f.265", "b_qcif_10f.265", "bbb1080_50f.265", "bbb1080_singleslice.265"])
def test_gpu_dropin_incremental_matches_batch(D, gpu_lib, name):
    _check(name, _decode_incremental(D, gpu_lib, name), "incremental")


@pytest.mark.gpu
@pytest.mark.parametrize("name", TEN_BIT)
def test_gpu_dropin_refuses_ten_bit(D, gpu_lib, name):
    dec = D.Decoder(gpu_lib)
    assert dec.decode(_data(name)) == -1
    assert "bit depth 10" in dec.last_error()
    assert dec.frames() == []
    dec.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["full_qcif_10f.265", "bbb1080_50f.265"])
def test_gpu_reference_cli_over_dropin(hb, gpu_lib, tmp_path, name):
    """The reference's own CLI (src/main.cpp: hevc::Decoder, output_pictures, write_yuv),
    linked against the drop-in library, writes the file the reference's test expects."""
    from hevc_b200 import build
    out = tmp_path / "out.yuv"
    r = subprocess.run([build.DROPIN_CLI, os.path.join(STREAMS, name), "-o", str(out)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert hashlib.md5(out.read_bytes()).hexdigest() == GOLDEN[name]["md5"]
