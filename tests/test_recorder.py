"""Real streams: privaloops/hevc.js decodes its own conformance and demo streams while
oracle/recorder.cpp records every picture as the records of include/hevcgpu.h (the
recorder of the integration plan, running inside the unmodified reference), and the
oracle must reconstruct each picture from those records exactly as the reference did.

This pins the record format and the oracle on real encoder output: I, P and B pictures,
explicit weighted prediction, SAO, deblocking, cu_qp_delta and scaling lists (bbb1080_50f).
It needs the reference tree (the streams) and oracle/_ref/hevc-record; it is skipped
without them.  10-bit streams are outside this path and are not run."""
import os
import subprocess

import pytest

import oracle

STREAMS = [os.path.join("tests", "conformance", "fixtures", f + ".265") for f in
           ("i_64x64_qp22", "i_64x64_full", "i_64x64_sao", "i_64x64_deblock", "toy_qp10", "toy_qp30", "toy_qp45",
            "i_qcif_176x144", "p_qcif_10f", "b_qcif_10f", "full_qcif_10f", "bbb1080_50f")] + \
          [os.path.join("demo", "bbb1080_singleslice.265")]


@pytest.mark.parametrize("stream", STREAMS)
def test_oracle_reconstructs_real_streams_from_recorded_records(stream):
    path = os.path.join(oracle.REF_DIR, stream)
    if not os.path.exists(path) or not os.path.exists(oracle.RECORDER):
        pytest.skip("needs the reference tree and oracle/_ref/hevc-record")
    r = subprocess.run([oracle.RECORDER, path], capture_output=True, text=True, timeout=600)
    lines = r.stdout.strip().splitlines()
    summary = lines[-1].split()
    # pictures N matched M mismatched K unsupported U decode_rc RC
    n, matched, mismatched, unsupported = int(summary[1]), int(summary[3]), int(summary[5]), int(summary[7])
    assert r.returncode == 0 and n > 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert mismatched == 0 and unsupported == 0 and matched == n, "\n".join(lines[-20:])
