"""The host intra schedule (hevcgpu_intra_schedule: the schedule k_intra_ctus runs, built
on the host) against a derivation of its own, on the CPU.

The derivation follows the reconstruction rule the schedule encodes: an intra TU reads the
reference row above it (x - 1 .. x + 2N - 1) and the column left of it (y .. y + 2N - 1),
intra_prediction.cpp:102-133, so it depends on the intra TUs decoded before it that own a
4x4 unit there, except those in CTUs later in raster order (never available,
intra_prediction.cpp:113).  Besides equal dependency sets, the test checks what makes the
kernel's waits safe: CTUs in wavefront order (key 2 * row + column), every local
dependency an earlier task of the same CTU, every watched TU a published task of an
earlier CTU."""
import numpy as np
import pytest

import cases

CONFIGS = {
    "I 416x240": dict(w=416, h=240, seed=3, cfg=dict(cases.ALL_INTRA, poc=0)),
    "P/B 1920x1080": dict(w=1920, h=1080, seed=1011, cfg=dict(cases.PICTURE, poc=8)),
    "I 352x288, 16x16 CTBs, 3x3 tiles": dict(w=352, h=288, seed=21,
                                             cfg=dict(cases.ALL_INTRA, poc=0, log2_ctb=4, tile_cols=3, tile_rows=3)),
    "P/B 416x240, 32x32 CTBs": dict(w=416, h=240, seed=17, cfg=dict(cases.PICTURE, poc=8, log2_ctb=5, p_intra=0.4)),
    "P/B 208x120, PCM": dict(w=208, h=120, seed=22, cfg=dict(cases.PICTURE, poc=8, p_intra=0.5, p_pcm=0.3)),
}


def derive(hb, pic):
    """(intra TU indices in decode order, CTU of each, set of dependencies of each), the
    dependencies as positions in the first list."""
    s = pic.syn
    prm = s.params
    W, H, lc = prm.width, prm.height, prm.log2_ctb
    wctb = (W + (1 << lc) - 1) >> lc
    tus = [s.tus[i] for i in range(s.num_tus)]
    intra = [i for i, t in enumerate(tus) if t.flags & hb.abi.HEVC_TU_INTRA]
    owner = [np.full(((H >> (1 if c else 0)) // 4, (W >> (1 if c else 0)) // 4), -1, np.int64) for c in range(3)]
    ctu, deps = [], []
    for b, i in enumerate(intra):
        t = tus[i]
        c, n, sub = t.c_idx, 1 << t.log2_size, 2 if t.c_idx else 1
        a = ((t.y * sub) >> lc) * wctb + ((t.x * sub) >> lc)
        ctu.append(a)
        o_map = owner[c]
        uh, uw = o_map.shape
        d = set()
        if t.y > 0:
            for ux in range(max(0, (t.x - 1) // 4), min(uw - 1, (t.x + 2 * n - 1) // 4) + 1):
                o = int(o_map[(t.y - 1) // 4, ux])
                if o >= 0 and ctu[o] <= a:
                    d.add(o)
        if t.x > 0:
            for uy in range(t.y // 4, min(uh - 1, (t.y + 2 * n - 1) // 4) + 1):
                o = int(o_map[uy, (t.x - 1) // 4])
                if o >= 0 and ctu[o] <= a:
                    d.add(o)
        deps.append(d)
        o_map[t.y // 4:(t.y + n) // 4, t.x // 4:(t.x + n) // 4] = b
    return intra, ctu, deps, wctb


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_intra_schedule_matches_its_derivation(hb, name):
    c = CONFIGS[name]
    pic = hb.Picture(hb.default_cfg(c["w"], c["h"], c["seed"], **c["cfg"]))
    sch = hb.intra_schedule(pic)
    intra, ctu, deps, wctb = derive(hb, pic)
    assert len(intra) > 0
    # every intra TU is one task; a task's TU lies in its CTU
    task_tu = sch["task_tu"]
    assert sorted(task_tu.tolist()) == intra
    b_of = {tu: b for b, tu in enumerate(intra)}
    first, addr = sch["ctu_first"], sch["ctu_addr"]
    assert first[0] == 0 and first[-1] == len(intra) and np.all(np.diff(first) > 0)
    assert len(set(addr.tolist())) == len(addr)
    keys = [2 * (a // wctb) + a % wctb for a in addr.tolist()]
    assert keys == sorted(keys), "CTUs in wavefront order"
    published = set(np.nonzero(sch["task_flags"] & hb.abi.HEVC_INTRA_PUBLISH)[0].tolist())
    watched = set()
    for k in range(len(addr)):
        w0, nw = int(sch["ctu_watch"][k]) >> 8, int(sch["ctu_watch"][k]) & 0xFF
        slots = sch["watch"][w0:w0 + nw].tolist()
        for task in slots:   # TUs of earlier CTUs, published by their tasks
            assert task < first[k] and task in published, (name, k, task)
        watched.update(slots)
        for j in range(int(first[k]), int(first[k + 1])):
            b = b_of[int(task_tu[j])]
            assert ctu[b] == addr[k]
            d0, nd = int(sch["task_deps"][j]) >> 6, int(sch["task_deps"][j]) & 63
            got = set()
            for e in sch["deps"][d0:d0 + nd].tolist():
                if e & hb.abi.HEVC_INTRA_DEP_WATCH:
                    slot = e & 0xFF
                    assert slot < nw
                    got.add(b_of[int(task_tu[slots[slot]])])
                else:
                    assert e < j - first[k], "a local dependency is an earlier task of the CTU"
                    got.add(b_of[int(task_tu[first[k] + e])])
            assert got == deps[b], (name, j)
    assert watched == published
