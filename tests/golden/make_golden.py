"""Generate tests/golden/digests.json from privaloops/hevc.js's own functions.

Runs every case of tests/cases.py through the reference harness (oracle/_ref, the
reference's transform.cpp / intra_prediction.cpp / interpolation.cpp / deblocking.cpp /
sao.cpp compiled from its sources by oracle/Makefile) and records per-plane MD5s of the
8-bit output, plus the realised Bs histogram of the filter cases.  Needs the reference
tree at build time only; the digests are committed.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))


def main():
    import __graft_entry__ as ge
    hb = ge.load_package()
    from hevc_b200 import build
    build.build_synth()
    import oracle
    oracle.build(with_ref=True)
    import cases
    ref = oracle.ref()
    out = {"generator": "tests/golden/make_golden.py", "checker": "oracle/_ref (reference sources)", "cases": {}}
    for name, case in cases.CASES.items():
        inp = cases.build_inputs(hb, case)
        res = cases.run_case(ref, case, inp)
        ent = {"md5": cases.digest(hb, case, res)}
        if case["kind"] in ("filters", "deblock"):
            ent["bs_histogram"] = inp["pic"].bs_histogram()
        if "pic" in inp:
            ent["counts"] = inp["pic"].counts()
        out["cases"][name] = ent
        print(name, ent["md5"][0], flush=True)
    with open(os.path.join(HERE, "digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
