"""ctypes mirror of include/hevcgpu.h and hevc.js_b200/csrc/synth.h.

The record layouts here must match the C headers byte for byte; the tests check the
sizes against the values the libraries report (``ctypes.sizeof`` against the C
``sizeof`` of each struct, which the libraries export through tiny size probes).
"""
import ctypes as C

import numpy as np

HEVCGPU_OK = 0
HEVCGPU_EINVAL = -1
HEVCGPU_ECUDA = -2
HEVCGPU_ENOMEM = -3
HEVCGPU_EUNSUPPORTED = -4
HEVCGPU_ETIMEOUT = -5
HEVCGPU_EDEVICE = -6

HEVC_TU_INTRA = 0x01
HEVC_TU_CODED = 0x02
HEVC_TU_TSKIP = 0x04
HEVC_TU_BYPASS = 0x08
HEVC_TU_PCM = 0x10

HEVC_BLK_EDGE_V = 0x01
HEVC_BLK_EDGE_H = 0x02
HEVC_BLK_CBF = 0x04
HEVC_BLK_INTRA = 0x08
HEVC_BLK_PCM = 0x10
HEVC_BLK_BYPASS = 0x20
HEVC_BLK_TU_SHIFT = 8
HEVC_BLK_QP_SHIFT = 16


class TU(C.Structure):
    _fields_ = [("x", C.c_uint16), ("y", C.c_uint16), ("log2_size", C.c_uint8), ("c_idx", C.c_uint8),
                ("qp", C.c_uint8), ("flags", C.c_uint8), ("intra_mode", C.c_uint8),
                ("reserved", C.c_uint8 * 3), ("coeff_offset", C.c_uint32)]


class PU(C.Structure):
    _fields_ = [("x", C.c_uint16), ("y", C.c_uint16), ("w", C.c_uint8), ("h", C.c_uint8),
                ("ref_idx", C.c_int8 * 2), ("mv", (C.c_int16 * 2) * 2), ("wp", C.c_int16),
                ("reserved", C.c_uint16)]


class WP(C.Structure):
    _fields_ = [("log2wd", C.c_int16 * 2), ("w", (C.c_int16 * 3) * 2), ("o", (C.c_int16 * 3) * 2)]


class SAO(C.Structure):
    _fields_ = [("type", C.c_uint8 * 3), ("band_pos", C.c_uint8 * 3), ("eo_class", C.c_uint8 * 3),
                ("offset", (C.c_int8 * 5) * 3)]


class Slice(C.Structure):
    _fields_ = [("beta_offset_div2", C.c_int8), ("tc_offset_div2", C.c_int8),
                ("deblocking_disabled", C.c_uint8), ("lf_across_slices", C.c_uint8)]


class Scaling(C.Structure):
    _fields_ = [("list", ((C.c_uint8 * 64) * 6) * 4), ("dc", (C.c_uint8 * 6) * 2), ("reserved", C.c_uint8 * 4)]


class Crop(C.Structure):
    _fields_ = [("left", C.c_int32), ("right", C.c_int32), ("top", C.c_int32), ("bottom", C.c_int32)]


HEVC_INTRA_DEP_WATCH = 0x40000000
HEVC_INTRA_PUBLISH = 1


class IntraSchedule(C.Structure):
    """hevc_intra_schedule_t: views into the calling thread's arrays (hevcgpu_intra_schedule)."""
    _fields_ = [("n_ctu", C.c_int32), ("n_task", C.c_int32), ("n_dep", C.c_int32), ("n_watch", C.c_int32),
                ("ctu_addr", C.POINTER(C.c_int32)), ("ctu_first", C.POINTER(C.c_int32)),
                ("task_tu", C.POINTER(C.c_int32)), ("task_deps", C.POINTER(C.c_uint32)),
                ("deps", C.POINTER(C.c_uint32)), ("task_flags", C.POINTER(C.c_uint8)),
                ("ctu_watch", C.POINTER(C.c_uint32)), ("watch", C.POINTER(C.c_uint32))]


class PicParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("bit_depth", C.c_int32),
                ("log2_ctb", C.c_int32), ("log2_min_cb", C.c_int32), ("log2_min_tb", C.c_int32),
                ("strong_intra_smoothing", C.c_int32), ("intra_smoothing_disabled", C.c_int32),
                ("pcm_loop_filter_disabled", C.c_int32), ("sao_enabled", C.c_int32),
                ("cb_qp_offset", C.c_int32), ("cr_qp_offset", C.c_int32),
                ("tiles_enabled", C.c_int32), ("loop_filter_across_tiles", C.c_int32),
                ("num_ref", C.c_int32 * 2), ("ref_poc", (C.c_int32 * 16) * 2),
                ("ref_slot", (C.c_int32 * 16) * 2)]


class PictureSyntax(C.Structure):
    _fields_ = [("params", PicParams),
                ("num_tus", C.c_int32), ("tus", C.POINTER(TU)),
                ("num_coeffs", C.c_uint64), ("coeffs", C.POINTER(C.c_int16)),
                ("num_pus", C.c_int32), ("pus", C.POINTER(PU)),
                ("num_wp", C.c_int32), ("wp", C.POINTER(WP)),
                ("blk", C.POINTER(C.c_uint32)),
                ("sao", C.POINTER(SAO)),
                ("ctb_slice", C.POINTER(C.c_uint8)),
                ("ctb_tile", C.POINTER(C.c_uint16)),
                ("num_slices", C.c_int32), ("slices", C.POINTER(Slice)),
                ("scaling", C.POINTER(Scaling))]


class SynthCfg(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("seed", C.c_uint64),
                ("p_split", C.c_double), ("p_intra", C.c_double), ("p_intra_nxn", C.c_double),
                ("p_skip", C.c_double), ("p_bi", C.c_double), ("p_wp", C.c_double),
                ("p_merge", C.c_double), ("mv_range", C.c_int32), ("p_tu_split", C.c_double),
                ("p_cbf_luma", C.c_double), ("p_cbf_chroma", C.c_double),
                ("qp_min", C.c_int32), ("qp_max", C.c_int32), ("sao", C.c_int32),
                ("num_refs", C.c_int32), ("slice_type", C.c_int32), ("poc", C.c_int32),
                ("strong_intra_smoothing", C.c_int32), ("cb_qp_offset", C.c_int32),
                ("cr_qp_offset", C.c_int32), ("beta_offset_div2", C.c_int32),
                ("tc_offset_div2", C.c_int32), ("scaling_lists", C.c_int32), ("log2_ctb", C.c_int32),
                ("tile_cols", C.c_int32), ("tile_rows", C.c_int32), ("no_lf_across_tiles", C.c_int32),
                ("p_pcm", C.c_double)]


class SynthCU(C.Structure):
    _fields_ = [("x", C.c_uint16), ("y", C.c_uint16), ("log2_size", C.c_uint8), ("pred_mode", C.c_uint8),
                ("part_mode", C.c_uint8), ("qp_y", C.c_int8), ("first_pu", C.c_int32),
                ("num_pu", C.c_int32), ("first_tu", C.c_int32), ("num_tu", C.c_int32),
                ("has_tree", C.c_int32), ("reserved", C.c_int32)]


class SynthPicture(C.Structure):
    _fields_ = [("syn", PictureSyntax), ("num_cus", C.c_int32), ("cus", C.POINTER(SynthCU)),
                ("impl", C.c_void_p)]


RECORD_SIZES = {"hevc_tu_t": 16, "hevc_pu_t": 20, "hevc_wp_t": 28, "hevc_sao_t": 24,
                "hevc_slice_t": 4, "hevc_scaling_t": 1552}


def check_layouts():
    got = {"hevc_tu_t": C.sizeof(TU), "hevc_pu_t": C.sizeof(PU), "hevc_wp_t": C.sizeof(WP),
           "hevc_sao_t": C.sizeof(SAO), "hevc_slice_t": C.sizeof(Slice), "hevc_scaling_t": C.sizeof(Scaling)}
    if got != RECORD_SIZES:
        raise AssertionError(f"record layout mismatch: {got} != {RECORD_SIZES}")


def i420_size(width, height):
    return width * height + 2 * (width // 2) * (height // 2)


def split_i420(buf, width, height):
    """Views of the Y, Cb, Cr planes of a packed I420 numpy buffer."""
    y = buf[: width * height].reshape(height, width)
    cw, ch = width // 2, height // 2
    cb = buf[width * height: width * height + cw * ch].reshape(ch, cw)
    cr = buf[width * height + cw * ch: width * height + 2 * cw * ch].reshape(ch, cw)
    return y, cb, cr


def as_ptr(arr, ctype):
    """ctypes pointer to the data of a contiguous numpy array (or None)."""
    if arr is None:
        return None
    assert arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(C.POINTER(ctype))


def ptr_array(bufs):
    """const uint8_t* const* from a list of numpy uint8 arrays."""
    arr = (C.POINTER(C.c_uint8) * len(bufs))()
    for i, b in enumerate(bufs):
        arr[i] = as_ptr(b, C.c_uint8)
    return arr


def md5_planes(buf, width, height):
    """Per-plane MD5 of an 8-bit I420 picture (the parity digest of the oracle tests)."""
    import hashlib
    return tuple(hashlib.md5(np.ascontiguousarray(p).tobytes()).hexdigest()
                 for p in split_i420(buf, width, height))
