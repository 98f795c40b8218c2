"""Make tests/golden/streams.json: what privaloops/hevc.js's own decoder outputs for the
conformance and demo streams under tests/golden/streams/.

The streams are the reference's test vectors (tests/conformance/fixtures/*.265 and
demo/bbb1080_singleslice.265), copied here so that tests run where the reference tree is
absent.  For each stream this script records, from the reference decoder built from its
own sources by oracle/Makefile (the reference tree must be present; HEVC_REF_DIR or a
checkout beside this repository):

  frames      per frame: POC and the MD5 of its samples as Picture::write_yuv writes them
              (src/common/picture.cpp:42-95), through the reference's C API
              (oracle/_ref/libhevcdec.so: its objects and its own src/wasm/hevc_api.cpp),
              in the order hevc_decoder_get_frame hands them out;
  md5         the MD5 of the whole output file of the reference's CLI (`hevc-decode in -o
              out.yuv`, src/main.cpp), which must equal the MD5 of the frames concatenated;
  published   the MD5 the reference's own test suite expects (CMakeLists.txt:139-224), when
              it has one; the script checks that the reference reproduces it;
  incremental per frame: POC and MD5 through hevc_decoder_feed per access unit, drain after
              each, and flush (the path of tests/unit/test_incremental.cpp:50-176).

Run: python tests/golden/make_streams_golden.py
"""
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import __graft_entry__ as ge  # noqa: E402

ge.load_package()
import oracle  # noqa: E402
from hevc_b200 import decoder as D  # noqa: E402

STREAMS = os.path.join(HERE, "streams")


def published_md5s(ref_dir):
    """fixture file name -> MD5 from the add_test(NAME oracle_* ...) lines of CMakeLists.txt."""
    text = open(os.path.join(ref_dir, "CMakeLists.txt")).read()
    out = {}
    for m in re.finditer(r"\$\{FIXTURES_DIR\}/(\S+\.265)\s+\d+\s+\d+\s*\n?\s*([0-9a-f]{32})", text):
        out[m.group(1)] = m.group(2)
    return out


def main():
    oracle.build()
    ref_lib = os.path.join(oracle.HERE, "_ref", "libhevcdec.so")
    pub = published_md5s(oracle.REF_DIR)
    golden = {}
    for name in sorted(os.listdir(STREAMS)):
        if not name.endswith(".265"):
            continue
        data = open(os.path.join(STREAMS, name), "rb").read()
        dec = D.Decoder(ref_lib)
        rc = dec.decode(data)
        assert rc == 0, (name, rc)
        frames = dec.frames()
        info = dec.info()
        dec.close()
        whole = hashlib.md5(b"".join(f.yuv_bytes() for f in frames)).hexdigest()
        with tempfile.TemporaryDirectory() as t:
            out = os.path.join(t, "out.yuv")
            subprocess.run([oracle.REF_CLI, os.path.join(STREAMS, name), "-o", out], check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            cli = hashlib.md5(open(out, "rb").read()).hexdigest()
        assert cli == whole, (name, cli, whole)
        if name in pub:
            assert pub[name] == whole, (name, "the reference does not reproduce its published MD5")
        inc = D.Decoder(ref_lib)
        inc_frames = []
        for chunk in D.split_access_units(data):
            assert inc.feed(chunk) == 0, name
            inc_frames += inc.drain()
        inc_frames += inc.flush()
        inc.close()
        golden[name] = {
            "width": info.width, "height": info.height, "bit_depth": info.bit_depth,
            "md5": whole, "published": pub.get(name),
            "frames": [[f.poc, f.md5()] for f in frames],
            "incremental": [[f.poc, f.md5()] for f in inc_frames],
        }
        print(f"{name}: {len(frames)} frames {info.width}x{info.height} {info.bit_depth}-bit md5 {whole}"
              f"{' (published)' if name in pub else ''}; incremental {len(inc_frames)} frames")
    with open(os.path.join(HERE, "streams.json"), "w") as f:
        json.dump(golden, f, indent=1)


if __name__ == "__main__":
    main()
