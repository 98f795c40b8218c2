"""The committed records of real streams (tests/golden/real/, made by
tests/golden/make_real_streams.py from privaloops/hevc.js decoding its own conformance
streams under oracle/recorder.cpp) replay through the oracle to the pictures the
reference decoded: every picture's MD5 equals the committed one.  Needs neither the
reference tree nor a GPU."""
import hashlib
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
STREAMS = json.load(open(os.path.join(GOLDEN, "real_streams.json")))["streams"]


@pytest.mark.parametrize("name", sorted(STREAMS))
def test_oracle_replays_recorded_real_streams(hb, port, name):
    import sys
    sys.path.insert(0, GOLDEN)
    import real_streams
    pics = real_streams.load(hb.abi, os.path.join(real_streams.DIR, name + ".hrec.xz"))
    want = STREAMS[name]
    assert len(pics) == want["pictures"]
    outs = real_streams.replay(port.reconstruct_picture, pics)
    assert [hashlib.md5(o.tobytes()).hexdigest() for o in outs] == want["md5"]
