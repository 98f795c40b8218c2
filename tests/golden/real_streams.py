"""Recorded real streams: the picture records oracle/recorder.cpp wrote while
privaloops/hevc.js decoded the reference's own conformance streams (format in
oracle/recorder.cpp), compressed with xz, and the MD5 of every picture.

load(path) gives the pictures in decode order; each picture's params name its references
by decode index (params.ref_slot).  replay(hb, reconstruct, pictures) reconstructs them in
order with `reconstruct(pic, refs)` (a checker's reconstruct_picture), every picture
predicted from the replay's own earlier outputs, and returns the outputs."""
import ctypes as C
import lzma
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DIR = os.path.join(HERE, "real")


class RecordedPicture:
    """A picture's records in numpy arrays and the PictureSyntax that points at them."""

    def __init__(self, abi, params, arrays, counts, has_scaling, has_tiles):
        self.arrays = arrays   # keeps the memory the syntax points to alive
        n_tus, n_coeffs, n_pus, n_wp, n_slices = (int(c) for c in counts)
        s = abi.PictureSyntax()
        s.params = params
        a = arrays
        s.num_tus = n_tus
        s.tus = a["tus"].ctypes.data_as(C.POINTER(abi.TU))
        s.num_coeffs = n_coeffs
        s.coeffs = a["coeffs"].ctypes.data_as(C.POINTER(C.c_int16))
        s.num_pus = n_pus
        s.pus = a["pus"].ctypes.data_as(C.POINTER(abi.PU))
        s.num_wp = n_wp
        s.wp = a["wp"].ctypes.data_as(C.POINTER(abi.WP))
        s.blk = a["blk"].ctypes.data_as(C.POINTER(C.c_uint32))
        s.sao = a["sao"].ctypes.data_as(C.POINTER(abi.SAO))
        s.ctb_slice = a["ctb_slice"].ctypes.data_as(C.POINTER(C.c_uint8))
        s.ctb_tile = a["ctb_tile"].ctypes.data_as(C.POINTER(C.c_uint16)) if has_tiles else None
        s.num_slices = n_slices
        s.slices = a["slices"].ctypes.data_as(C.POINTER(abi.Slice))
        s.scaling = a["scaling"].ctypes.data_as(C.POINTER(abi.Scaling)) if has_scaling else None
        self.syn = s

    @property
    def syn_ptr(self):
        return C.pointer(self.syn)

    @property
    def width(self):
        return self.syn.params.width

    @property
    def height(self):
        return self.syn.params.height


def load(abi, path):
    raw = lzma.decompress(open(path, "rb").read()) if path.endswith(".xz") else open(path, "rb").read()
    assert raw[:4] == b"HREC" and int.from_bytes(raw[4:8], "little") == 1, path
    pos, pics = 8, []

    def take(n, dtype=np.uint8):
        nonlocal pos
        b = np.frombuffer(raw, dtype=np.uint8, count=n, offset=pos).copy()
        pos += n
        return b.view(dtype) if dtype is not np.uint8 else b

    while pos < len(raw):
        params = abi.PicParams.from_buffer_copy(raw, pos)
        pos += C.sizeof(abi.PicParams)
        n_tus, n_coeffs, n_pus, n_wp, n_slices = np.frombuffer(raw, np.int32, 5, pos)
        pos += 20
        has_scaling, has_tiles = raw[pos], raw[pos + 1]
        pos += 4
        W, H, ctb = params.width, params.height, 1 << params.log2_ctb
        nctb = ((W + ctb - 1) // ctb) * ((H + ctb - 1) // ctb)
        a = {"tus": take(16 * n_tus), "coeffs": take(2 * n_coeffs, np.int16), "pus": take(20 * n_pus),
             "wp": take(C.sizeof(abi.WP) * n_wp), "blk": take(4 * (W // 4) * (H // 4), np.uint32),
             "sao": take(C.sizeof(abi.SAO) * nctb), "ctb_slice": take(nctb)}
        a["ctb_tile"] = take(2 * nctb, np.uint16) if has_tiles else None
        a["slices"] = take(C.sizeof(abi.Slice) * n_slices)
        a["scaling"] = take(C.sizeof(abi.Scaling)) if has_scaling else None
        pics.append(RecordedPicture(abi, params, a, (n_tus, n_coeffs, n_pus, n_wp, n_slices), has_scaling, has_tiles))
    return pics


def replay(reconstruct, pictures):
    outs = []
    for pic in pictures:
        outs.append(reconstruct(pic, outs if outs else [np.zeros(1, np.uint8)]))
    return outs
