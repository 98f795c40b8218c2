"""Seeded parity cases shared by the golden-vector generator and the tests.

Every case is rebuilt from its seed by the package's generator, so the GPU box only
needs the committed digests (tests/golden/digests.json), never the reference tree.
"""
import numpy as np

# Generator settings per workload (see hevc.js_b200/csrc/synth.h for the knobs).
INTER = dict(p_intra=0.0, sao=0)                                   # inter prediction, 1080p
FILTERS = dict(p_intra=0.1, p_merge=0.95, p_cbf_luma=0.15, p_skip=0.8)   # Bs ~ 0.5/0.3/0.2
PICTURE = dict(p_intra=0.1, p_skip=0.2, p_merge=0.3)               # full P/B-like picture
INTRA_HEAVY = dict(p_intra=0.5)
ALL_INTRA = dict(slice_type=2)

CASES = {
    # config 1: 4096 independent residual blocks
    "blocks_4096_s0": dict(kind="blocks", n=4096, seed=0),
    "blocks_512_s7": dict(kind="blocks", n=512, seed=7),
    # config 2: inter prediction of a 1080p picture from two references
    "inter_1080p_s1": dict(kind="inter", w=1920, h=1080, seed=1, cfg=INTER, refs=(101, 102)),
    "inter_208x120_s8": dict(kind="inter", w=208, h=120, seed=8, cfg=dict(INTER, mv_range=2048), refs=(81, 82)),
    # config 3: deblocking + SAO at 1080p and 2160p
    "filters_1080p_s2": dict(kind="filters", w=1920, h=1080, seed=2, cfg=FILTERS, content=2),
    "filters_2160p_s2": dict(kind="filters", w=3840, h=2160, seed=2, cfg=FILTERS, content=3),
    "deblock_1080p_s2": dict(kind="deblock", w=1920, h=1080, seed=2, cfg=FILTERS, content=2),
    "filters_200x120_s9": dict(kind="filters", w=200, h=120, seed=9, cfg=FILTERS, content=4),
    # intra wavefront over an inter picture
    "intra_416x240_s5": dict(kind="intra", w=416, h=240, seed=5, cfg=INTRA_HEAVY, content=9),
    # whole pictures
    "picture_416x240_s3": dict(kind="picture", w=416, h=240, seed=3, cfg=PICTURE, refs=(31, 32)),
    "picture_1080p_s4": dict(kind="picture", w=1920, h=1080, seed=4, cfg=PICTURE, refs=(41, 42)),
    "picture_intra_352x288_s6": dict(kind="picture", w=352, h=288, seed=6, cfg=ALL_INTRA, refs=(61, 62)),
    "picture_64x64_s10": dict(kind="picture", w=64, h=64, seed=10, cfg=PICTURE, refs=(101, 102)),
    "picture_72x40_s12": dict(kind="picture", w=72, h=40, seed=12, cfg=dict(PICTURE, p_intra=0.4), refs=(121, 122)),
    # scaling lists (scaling_list_enabled_flag): blocks of every matrix, and whole pictures
    "blocks_scaled_2048_s13": dict(kind="blocks", n=2048, seed=13, scaling=113, mix=True),
    "picture_scaled_416x240_s14": dict(kind="picture", w=416, h=240, seed=14,
                                       cfg=dict(PICTURE, p_intra=0.3, scaling_lists=1), refs=(141, 142)),
    "picture_scaled_1080p_s15": dict(kind="picture", w=1920, h=1080, seed=15, cfg=dict(PICTURE, scaling_lists=1),
                                     refs=(151, 152)),
    # 16x16 and 32x32 CTBs (CtbLog2SizeY 4 and 5)
    "picture_ctb16_352x288_s16": dict(kind="picture", w=352, h=288, seed=16, cfg=dict(PICTURE, log2_ctb=4),
                                      refs=(161, 162)),
    "picture_ctb32_416x240_s17": dict(kind="picture", w=416, h=240, seed=17,
                                      cfg=dict(PICTURE, log2_ctb=5, p_intra=0.4), refs=(171, 172)),
    "picture_intra_ctb16_208x120_s18": dict(kind="picture", w=208, h=120, seed=18, cfg=dict(ALL_INTRA, log2_ctb=4),
                                            refs=(181, 182)),
    # tiles (uniform spacing, CTBs in tile scan), with and without filtering across them
    "picture_tiles_416x240_s19": dict(kind="picture", w=416, h=240, seed=19,
                                      cfg=dict(PICTURE, p_intra=0.4, tile_cols=3, tile_rows=2), refs=(191, 192)),
    "picture_tiles_1080p_s20": dict(kind="picture", w=1920, h=1080, seed=20,
                                    cfg=dict(PICTURE, tile_cols=4, tile_rows=3, no_lf_across_tiles=1), refs=(201, 202)),
    "picture_pcm_416x240_s22": dict(kind="picture", w=416, h=240, seed=22, cfg=dict(PICTURE, p_intra=0.5, p_pcm=0.3),
                                    refs=(221, 222)),
    "picture_intra_tiles_ctb16_352x288_s21": dict(kind="picture", w=352, h=288, seed=21,
                                                  cfg=dict(ALL_INTRA, log2_ctb=4, tile_cols=4, tile_rows=3,
                                                           no_lf_across_tiles=1), refs=(211, 212)),
}


def mix_blocks(hb, tus, n, seed, qp=(0, 51)):
    """Spread blocks over every scaling matrix: intra or not, any plane below 32x32, QP
    uniform in qp (None: kept)."""
    rng = np.random.default_rng(seed)
    for i in range(n):
        if rng.random() < 0.5:
            tus[i].flags ^= hb.abi.HEVC_TU_INTRA
        if tus[i].log2_size < 5:
            tus[i].c_idx = int(rng.integers(0, 3))
        if qp is not None:
            tus[i].qp = int(rng.integers(qp[0], qp[1] + 1))


def build_inputs(hb, case):
    """Inputs of a case: dict with the generated picture / blocks and sample buffers."""
    k = case["kind"]
    if k == "blocks":
        tus, n, coeffs, pred = hb.blocks(case["n"], case["seed"])
        if case.get("mix"):
            mix_blocks(hb, tus, n, case["seed"])
        sl = hb.scaling(case["scaling"]) if "scaling" in case else None
        return dict(tus=tus, n=n, coeffs=coeffs, pred=pred, scaling=sl)
    cfg = hb.default_cfg(case["w"], case["h"], case["seed"], **case["cfg"])
    pic = hb.Picture(cfg)
    out = dict(pic=pic)
    if "refs" in case:
        out["refs"] = [hb.content(case["w"], case["h"], s) for s in case["refs"]]
    if "content" in case:
        out["content"] = hb.content(case["w"], case["h"], case["content"])
    return out


def run_case(checker, case, inp):
    """Run a case through any object with the stage entry points (GPU context or oracle)."""
    k = case["kind"]
    if k == "blocks":
        return checker.residual_blocks(inp["tus"], inp["n"], inp["coeffs"], inp["pred"], inp["scaling"])
    if k == "inter":
        return checker.inter_pred(inp["pic"], inp["refs"])
    if k == "filters":
        return checker.loop_filter(inp["pic"], inp["content"], True, True)
    if k == "deblock":
        return checker.loop_filter(inp["pic"], inp["content"], True, False)
    if k == "intra":
        return checker.intra_recon(inp["pic"], inp["content"])
    if k == "picture":
        return checker.reconstruct_picture(inp["pic"], inp["refs"])
    raise KeyError(k)


def digest(hb, case, out):
    if case["kind"] == "blocks":
        import hashlib
        return [hashlib.md5(np.ascontiguousarray(out).tobytes()).hexdigest()]
    return list(hb.md5_planes(out, case["w"], case["h"]))


def picture_checksum(plane):
    """The checksum of the H.265 decoded picture hash SEI (Rec. ITU-T H.265 D.3.19) of one
    8-bit plane: the sum modulo 2^32 of sample ^ ((x & 0xFF) ^ (y & 0xFF) ^ (x >> 8) ^
    (y >> 8)), x and y counted from the plane's top-left corner."""
    h, w = plane.shape
    x = np.arange(w, dtype=np.uint32)
    y = np.arange(h, dtype=np.uint32)
    mask = ((x & 0xFF) ^ (x >> 8))[None, :] ^ ((y & 0xFF) ^ (y >> 8))[:, None]
    return int(((plane.astype(np.uint32) & 0xFF) ^ mask).sum(dtype=np.uint64) & 0xFFFFFFFF)
