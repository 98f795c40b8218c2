"""Python mirror of the hevc.js decoder C API with reconstruction on the GPU.

``libhevcdec_gpu.so`` (include/hevc_api_gpu.h) exports the reference's decoder API
(privaloops/hevc.js src/wasm/hevc_api.h:13-86): the reference's host parser with the
reconstruction hooks recording, and every picture reconstructed by ``libhevcgpu.so``.
``Decoder`` binds those exports with ctypes, as the reference's TypeScript binding binds
them through cwrap (packages/core/src/decoder.ts), and hands frames out as numpy planes.

The same class binds any library with the reference's exports: the tests also load the
reference's own build of its API and a checker build (test infrastructure) to compare
against.  ``split_access_units`` cuts an Annex B stream into the complete access units
the incremental calls (feed/drain/flush, hevc_api.h:68-84) take.
"""
import ctypes as C
import hashlib
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
DROPIN_SO = os.path.join(PKG, "libhevcdec_gpu.so")

HEVC_OK = 0
HEVC_ERROR = -1


class HEVCFrame(C.Structure):
    """hevc_api.h:21-33."""
    _fields_ = [("y", C.POINTER(C.c_uint16)), ("cb", C.POINTER(C.c_uint16)), ("cr", C.POINTER(C.c_uint16)),
                ("width", C.c_int), ("height", C.c_int), ("stride_y", C.c_int), ("stride_c", C.c_int),
                ("chroma_width", C.c_int), ("chroma_height", C.c_int), ("bit_depth", C.c_int), ("poc", C.c_int)]


class HEVCStreamInfo(C.Structure):
    """hevc_api.h:35-42."""
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("bit_depth", C.c_int), ("chroma_format", C.c_int),
                ("profile", C.c_int), ("level", C.c_int)]


class Frame:
    """A frame copied out of decoder-owned memory: 16-bit planes inside the conformance window."""

    def __init__(self, f):
        self.width, self.height, self.poc, self.bit_depth = f.width, f.height, f.poc, f.bit_depth
        self.planes = []
        for ptr, w, h, stride in ((f.y, f.width, f.height, f.stride_y),
                                  (f.cb, f.chroma_width, f.chroma_height, f.stride_c),
                                  (f.cr, f.chroma_width, f.chroma_height, f.stride_c)):
            a = np.ctypeslib.as_array(ptr, shape=(max(h - 1, 0) * stride + w,)) if h > 0 and w > 0 else np.zeros(0, np.uint16)
            rows = [a[r * stride:r * stride + w] for r in range(h)]
            self.planes.append(np.array(rows, dtype=np.uint16).reshape(h, w))

    def yuv_bytes(self):
        """The frame as Picture::write_yuv writes it (src/common/picture.cpp:42-95): 8-bit
        samples narrowed to bytes, deeper ones as little-endian 16-bit words."""
        if self.bit_depth <= 8:
            return b"".join(p.astype(np.uint8).tobytes() for p in self.planes)
        return b"".join(p.astype("<u2").tobytes() for p in self.planes)

    def md5(self):
        return hashlib.md5(self.yuv_bytes()).hexdigest()


def _bind(lib):
    vp = C.c_void_p
    sigs = {
        "hevc_decoder_create": ([], vp),
        "hevc_decoder_destroy": ([vp], None),
        "hevc_decoder_decode": ([vp, C.c_char_p, C.c_size_t], C.c_int),
        "hevc_decoder_get_frame_count": ([vp], C.c_int),
        "hevc_decoder_get_frame": ([vp, C.c_int, C.POINTER(HEVCFrame)], C.c_int),
        "hevc_decoder_get_info": ([vp, C.POINTER(HEVCStreamInfo)], C.c_int),
        "hevc_decoder_feed": ([vp, C.c_char_p, C.c_size_t], C.c_int),
        "hevc_decoder_drain": ([vp, C.POINTER(C.c_int)], C.c_int),
        "hevc_decoder_get_drained_frame": ([vp, C.c_int, C.POINTER(HEVCFrame)], C.c_int),
        "hevc_decoder_flush": ([vp], C.c_int),
    }
    for name, (args, res) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    if hasattr(lib, "hevc_decoder_last_error"):   # additions of libhevcdec_gpu.so
        lib.hevc_decoder_last_error.argtypes = [vp]
        lib.hevc_decoder_last_error.restype = C.c_char_p
        lib.hevc_decoder_set_device.argtypes = [vp, C.c_int]
        lib.hevc_decoder_set_device.restype = C.c_int
        lib.hevc_decoder_gpu_stats.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        lib.hevc_decoder_gpu_stats.restype = C.c_int
        lib.hevc_decoder_gpu_wait_ns.argtypes = [vp, C.POINTER(C.c_uint64)]
        lib.hevc_decoder_gpu_wait_ns.restype = C.c_int
    return lib


_libs = {}


def load(path=None):
    path = os.path.abspath(path or DROPIN_SO)
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (hevc.js_b200/build.py builds it from the reference's "
                                    f"parser sources)")
        _libs[path] = _bind(C.CDLL(path))
    return _libs[path]


class Decoder:
    """One decoder instance of the C API; ``lib`` is a library path (default: the GPU drop-in)."""

    def __init__(self, lib=None, device=None):
        self.lib = load(lib)
        self.h = self.lib.hevc_decoder_create()
        if not self.h:
            raise MemoryError("hevc_decoder_create")
        if device is not None:
            if self.lib.hevc_decoder_set_device(self.h, int(device)) != HEVC_OK:
                raise RuntimeError("hevc_decoder_set_device")

    def close(self):
        if self.h:
            self.lib.hevc_decoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self):
        if hasattr(self.lib, "hevc_decoder_last_error"):
            return (self.lib.hevc_decoder_last_error(self.h) or b"").decode()
        return ""

    def gpu_stats(self):
        p, n = C.c_uint64(0), C.c_uint64(0)
        self.lib.hevc_decoder_gpu_stats(self.h, C.byref(p), C.byref(n))
        return p.value, n.value

    def gpu_wait_ns(self):
        """Nanoseconds the decoder's calls have waited for the GPU back end."""
        ns = C.c_uint64(0)
        self.lib.hevc_decoder_gpu_wait_ns(self.h, C.byref(ns))
        return ns.value

    def decode(self, data):
        return self.lib.hevc_decoder_decode(self.h, bytes(data), len(data))

    def frames(self):
        out = []
        f = HEVCFrame()
        for i in range(self.lib.hevc_decoder_get_frame_count(self.h)):
            if self.lib.hevc_decoder_get_frame(self.h, i, C.byref(f)) != HEVC_OK:
                raise RuntimeError(f"hevc_decoder_get_frame({i})")
            out.append(Frame(f))
        return out

    def info(self):
        i = HEVCStreamInfo()
        return i if self.lib.hevc_decoder_get_info(self.h, C.byref(i)) == HEVC_OK else None

    def feed(self, data):
        return self.lib.hevc_decoder_feed(self.h, bytes(data), len(data))

    def _drained(self, n):
        out = []
        f = HEVCFrame()
        for i in range(n):
            if self.lib.hevc_decoder_get_drained_frame(self.h, i, C.byref(f)) != HEVC_OK:
                raise RuntimeError(f"hevc_decoder_get_drained_frame({i})")
            out.append(Frame(f))
        return out

    def drain(self):
        n = C.c_int(0)
        if self.lib.hevc_decoder_drain(self.h, C.byref(n)) != HEVC_OK:
            raise RuntimeError("hevc_decoder_drain: " + self.last_error())
        return self._drained(n.value)

    def flush(self):
        if self.lib.hevc_decoder_flush(self.h) != HEVC_OK:
            raise RuntimeError("hevc_decoder_flush: " + self.last_error())
        n = C.c_int(0)
        # flush leaves the remaining pictures in the drained list (hevc_api.cpp:164-174)
        f = HEVCFrame()
        out = []
        i = 0
        while self.lib.hevc_decoder_get_drained_frame(self.h, i, C.byref(f)) == HEVC_OK:
            out.append(Frame(f))
            i += 1
        del n
        return out


def _nal_units(data):
    """(start, end) of each NAL unit's payload in an Annex B byte stream."""
    b = bytes(data)
    starts = []
    i, n = 0, len(b)
    while i + 3 <= n:
        if b[i] == 0 and b[i + 1] == 0 and b[i + 2] == 1:
            starts.append(i + 3)
            i += 3
        else:
            i += 1
    out = []
    for k, s in enumerate(starts):
        e = starts[k + 1] - 3 if k + 1 < len(starts) else n
        while e > s and b[e - 1] == 0:   # the leading zero of a 4-byte start code
            e -= 1
        out.append((s, e))
    return out


def split_access_units(data):
    """Chunks of complete access units: each ends where the next picture's first NAL unit
    begins (a non-VCL unit after a VCL one, or a VCL unit with first_slice_segment_in_pic_flag),
    so no picture's slices are split between two feed calls."""
    b = bytes(data)
    nals = _nal_units(b)
    chunks, begin, seen_vcl = [], 0, False
    for s, e in nals:
        if e - s < 3:
            continue
        typ = (b[s] >> 1) & 0x3F
        vcl = typ < 32
        first_slice = vcl and (b[s + 2] & 0x80) != 0
        if seen_vcl and (not vcl or first_slice):
            cut = s - 3
            while cut > begin and b[cut - 1] == 0:
                cut -= 1
            chunks.append(b[begin:cut])
            begin, seen_vcl = cut, False
        seen_vcl = seen_vcl or vcl
    chunks.append(b[begin:])
    return [c for c in chunks if c]
