"""The seeded workload generator: deterministic, legal-shaped, and faithful to the
distributions the workloads name."""
import numpy as np

import cases


def _tu_array(hb, pic):
    s = pic.syn
    return [s.tus[i] for i in range(s.num_tus)]


def test_generator_is_deterministic(hb):
    a = hb.Picture(hb.default_cfg(416, 240, 5, **cases.PICTURE))
    b = hb.Picture(hb.default_cfg(416, 240, 5, **cases.PICTURE))
    assert a.counts() == b.counts()
    na = a.syn.num_coeffs
    ca = np.ctypeslib.as_array(a.syn.coeffs, (na,))
    cb = np.ctypeslib.as_array(b.syn.coeffs, (na,))
    assert np.array_equal(ca, cb)
    assert np.array_equal(hb.content(64, 32, 3), hb.content(64, 32, 3))


def test_records_stay_inside_the_picture(hb):
    for seed, (w, h) in enumerate([(1920, 1080), (200, 120), (72, 40)]):
        pic = hb.Picture(hb.default_cfg(w, h, seed, **cases.PICTURE))
        s = pic.syn
        for t in _tu_array(hb, pic):
            n = 1 << t.log2_size
            sub = 2 if t.c_idx else 1
            assert t.x % n == 0 and t.y % n == 0 and t.x + n <= w // sub and t.y + n <= h // sub
            assert t.coeff_offset % 16 == 0
        for i in range(s.num_pus):
            u = s.pus[i]
            assert u.x + u.w <= w and u.y + u.h <= h and (u.ref_idx[0] >= 0 or u.ref_idx[1] >= 0)
            if u.w + u.h == 12:
                assert not (u.ref_idx[0] >= 0 and u.ref_idx[1] >= 0)


def test_pus_tile_the_inter_area(hb):
    w, h = 320, 192
    pic = hb.Picture(hb.default_cfg(w, h, 3, p_intra=0.0))
    cover = np.zeros((h, w), np.int32)
    s = pic.syn
    for i in range(s.num_pus):
        u = s.pus[i]
        cover[u.y:u.y + u.h, u.x:u.x + u.w] += 1
    assert (cover == 1).all()


def test_block_mix_and_levels(hb):
    tus, n, coeffs, pred = hb.blocks(4096, 0)
    sizes = np.array([tus[i].log2_size for i in range(n)])
    dst = np.array([tus[i].flags & hb.abi.HEVC_TU_INTRA for i in range(n)]) != 0
    frac = [np.mean(dst), np.mean((sizes == 2) & ~dst), np.mean(sizes == 3), np.mean(sizes == 4), np.mean(sizes == 5)]
    for f, want in zip(frac, [0.25, 0.25, 0.25, 0.15, 0.10]):
        assert abs(f - want) < 0.03
    qps = np.array([tus[i].qp for i in range(n)])
    assert qps.min() >= 22 and qps.max() <= 37
    assert np.abs(coeffs).max() >= 2 and (coeffs != 0).mean() < 0.5
