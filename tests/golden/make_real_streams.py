"""Generate tests/golden/real/: records of the reference's own 8-bit conformance streams,
written by oracle/recorder.cpp while privaloops/hevc.js decodes them (every picture is
checked there: the oracle rebuilds it from its records exactly as the reference does),
xz-compressed, and real_streams.json with the MD5 of every picture, taken from the
oracle's replay of the records.  Needs the reference tree at build time only.

    python tests/golden/make_real_streams.py
"""
import hashlib
import json
import lzma
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

STREAMS = ["i_64x64_sao", "i_64x64_deblock", "toy_qp30", "i_qcif_176x144", "p_qcif_10f", "b_qcif_10f",
           "full_qcif_10f"]


def fnv64(a):
    h = 1469598103934665603
    for v in a.tobytes():
        h = ((h ^ v) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


def main():
    import __graft_entry__ as ge
    hb = ge.load_package()
    import oracle
    oracle.build(with_ref=True)
    import real_streams
    port = oracle.port()
    os.makedirs(real_streams.DIR, exist_ok=True)
    out = {"generator": "tests/golden/make_real_streams.py", "recorder": "oracle/recorder.cpp", "streams": {}}
    for name in STREAMS:
        src = os.path.join(oracle.REF_DIR, "tests", "conformance", "fixtures", name + ".265")
        with tempfile.TemporaryDirectory() as tmp:
            dump = os.path.join(tmp, name + ".hrec")
            r = subprocess.run([oracle.RECORDER, src, dump], capture_output=True, text=True, check=True)
            lines = r.stdout.strip().splitlines()
            summary = lines[-1].split()
            assert int(summary[5]) == 0 and int(summary[7]) == 0, r.stdout
            fnv_ref = [ln.split()[-1] for ln in lines[:-1] if ": match" in ln]
            raw = open(dump, "rb").read()
        dst = os.path.join(real_streams.DIR, name + ".hrec.xz")
        open(dst, "wb").write(lzma.compress(raw, preset=9 | lzma.PRESET_EXTREME))
        pics = real_streams.load(hb.abi, dst)
        outs = real_streams.replay(port.reconstruct_picture, pics)
        assert [fnv64(o) for o in outs] == fnv_ref, name   # the replay gives the reference's pictures
        out["streams"][name] = {"pictures": len(pics), "size": [pics[0].width, pics[0].height],
                                "md5": [hashlib.md5(o.tobytes()).hexdigest() for o in outs]}
        print(name, len(pics), os.path.getsize(dst), flush=True)
    with open(os.path.join(HERE, "real_streams.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
