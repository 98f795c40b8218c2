"""ctypes binding of the random-syntax bitstream generator (csrc/bitgen.h).

``generate(width, height, seed, **cfg)`` returns the Annex-B byte stream (an IDR picture,
then IDR pictures or, with ``inter=1``, low-delay P and B pictures) and, per picture, the
records the generator drew: the TUs (``hevc_tu_t``: every TU of an intra CU, the coded ones
of an inter CU) with their level pool, and the PUs (``hevc_pu_t``: position and size; an
AMVP-coded PU's ref_idx and coded mvd; -2 in ref_idx for a merged or skipped PU).  That is
what a recorder inside the reference decoder sees when it parses the stream, up to the
motion the decoder derives."""
import collections
import ctypes as C
import os

import numpy as np

from . import abi

PKG = os.path.dirname(os.path.abspath(__file__))
BITGEN_SO = os.path.join(PKG, "libhevcbitgen.so")


class GenCfg(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("seed", C.c_uint64), ("pictures", C.c_int32),
                ("log2_ctb", C.c_int32), ("p_split", C.c_double), ("p_nxn", C.c_double), ("p_tu_split", C.c_double),
                ("p_cbf", C.c_double), ("p_sig", C.c_double), ("max_level", C.c_int32), ("qp_min", C.c_int32),
                ("qp_max", C.c_int32), ("sao", C.c_int32), ("inter", C.c_int32), ("p_b", C.c_double),
                ("max_refs", C.c_int32), ("p_intra_cu", C.c_double), ("p_skip", C.c_double),
                ("p_merge", C.c_double), ("max_mvd", C.c_int32), ("amp", C.c_int32), ("tmvp", C.c_int32),
                ("max_merge", C.c_int32), ("wp", C.c_int32), ("depth_inter", C.c_int32),
                ("qp_delta_depth", C.c_int32), ("chroma_qp_offsets", C.c_int32), ("deblock_ctl", C.c_int32),
                ("slices", C.c_int32), ("dependent_slices", C.c_int32), ("tile_cols", C.c_int32), ("tile_rows", C.c_int32), ("wpp", C.c_int32),
                ("p_bypass", C.c_double), ("p_tskip", C.c_double), ("sdh", C.c_int32), ("p_pcm", C.c_double),
                ("scaling", C.c_int32), ("ref_quirks", C.c_int32), ("ra_gop", C.c_int32),
                ("idr_period", C.c_int32), ("crop", C.c_int32), ("p_no_output", C.c_double),
                ("long_term", C.c_int32), ("list_mod", C.c_int32), ("extra_syntax", C.c_int32),
                ("sps_rps", C.c_int32), ("cra", C.c_int32), ("poc_lsb_bits", C.c_int32),
                ("resize", C.c_int32), ("temporal", C.c_int32), ("nonref_types", C.c_int32),
                ("pps_count", C.c_int32), ("bit_depth", C.c_int32)]

# ref_quirks bits (csrc/bitgen.h): tools written the way the reference's parser reads them
QUIRK_TILES_PCM, QUIRK_DEPENDENT = 1, 2


class GenStream(C.Structure):
    _fields_ = [("bytes", C.POINTER(C.c_uint8)), ("size", C.c_size_t), ("pictures", C.c_int32),
                ("num_tus", C.POINTER(C.c_int32)), ("tus", C.POINTER(C.POINTER(abi.TU))),
                ("num_coeffs", C.POINTER(C.c_uint64)), ("coeffs", C.POINTER(C.POINTER(C.c_int16))),
                ("slice_type", C.POINTER(C.c_int32)), ("poc", C.POINTER(C.c_int32)),
                ("output", C.POINTER(C.c_int32)), ("tid", C.POINTER(C.c_int32)), ("crop", C.c_int32 * 4),
                ("num_pus", C.POINTER(C.c_int32)),
                ("pus", C.POINTER(C.POINTER(abi.PU)))]

# slice_type values (7.4.7.1)
SLICE_B, SLICE_P, SLICE_I = 0, 1, 2

GenPicture = collections.namedtuple("GenPicture", "tus levels pus slice_type poc output tid")


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(BITGEN_SO):
            raise RuntimeError(f"{BITGEN_SO} is not built (run __graft_entry__.build())")
        _lib = C.CDLL(BITGEN_SO)
        _lib.hevcgen_default_cfg.argtypes = [C.POINTER(GenCfg), C.c_int32, C.c_int32, C.c_uint64]
        _lib.hevcgen_default_cfg.restype = None
        _lib.hevcgen_stream.argtypes = [C.POINTER(GenCfg)]
        _lib.hevcgen_stream.restype = C.POINTER(GenStream)
        _lib.hevcgen_stream_free.argtypes = [C.POINTER(GenStream)]
        _lib.hevcgen_stream_free.restype = None
    return _lib


def generate(width, height, seed, **cfg):
    """(stream bytes, [GenPicture per picture, in decode order])."""
    g = lib()
    c = GenCfg()
    g.hevcgen_default_cfg(C.byref(c), width, height, seed)
    for k, v in cfg.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    sp = g.hevcgen_stream(C.byref(c))
    if not sp:
        raise ValueError("hevcgen_stream: bad configuration")
    try:
        s = sp.contents
        data = C.string_at(s.bytes, s.size)
        pics = []
        for k in range(s.pictures):
            tus = [abi.TU.from_buffer_copy(s.tus[k][i]) for i in range(s.num_tus[k])]
            n = int(s.num_coeffs[k])
            levels = np.ctypeslib.as_array(s.coeffs[k], shape=(n,)).copy() if n else np.zeros(0, np.int16)
            pus = [abi.PU.from_buffer_copy(s.pus[k][i]) for i in range(s.num_pus[k])]
            pics.append(GenPicture(tus, levels, pus, int(s.slice_type[k]), int(s.poc[k]), bool(s.output[k]),
                                   int(s.tid[k])))
        return data, pics
    finally:
        g.hevcgen_stream_free(sp)
