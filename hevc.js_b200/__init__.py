"""hevc.js B200 reconstruction back end — Python host mirror of the C ABI.

The product is the C-ABI library ``libhevcgpu.so`` (include/hevcgpu.h): the hevc.js
decoder's reconstruction path (dequant + inverse transform, intra and inter
prediction, deblocking, SAO, DPB in HBM) as sm_100a CUDA kernels.  This module binds it
with ctypes so that Python tests and benchmarks call exactly the entry points a C/C++
host calls.  It has no compute of its own and no CPU fallback: when the library or a
CUDA device is missing, ``Context()`` raises.

The stage functions mirror the reference's hot-path functions (privaloops/hevc.js):

  Context.residual_blocks      perform_dequant + perform_transform_inverse +
                               reconstruct_block  (src/decoding/transform.cpp:293, :374;
                               src/decoding/coding_tree.cpp:371)
  Context.inter_pred           perform_inter_prediction (src/decoding/interpolation.cpp:306)
  Context.intra_recon          perform_intra_prediction (src/decoding/intra_prediction.cpp:428)
  Context.loop_filter          apply_deblocking + apply_sao (src/filters/deblocking.cpp:357,
                               src/filters/sao.cpp:20)
  Context.reconstruct_picture  the per-picture reconstruction of Decoder::decode_picture
                               (src/decoding/decoder.cpp:52-304) minus parsing

Errors follow the reference C API (src/wasm/hevc_api.h:43-45): a negative status is an
error; here it is raised as ``HevcGpuError`` carrying the library's message.
"""
import ctypes as C
import os
import weakref

import numpy as np

from . import abi
from .abi import (TU, PU, WP, SAO, Slice, Scaling, PicParams, PictureSyntax, SynthCfg, SynthPicture,
                  i420_size, split_i420, as_ptr, ptr_array, md5_planes)

PKG = os.path.dirname(os.path.abspath(__file__))
SYNTH_SO = os.path.join(PKG, "libhevcsynth.so")
GPU_SO = os.path.join(PKG, "libhevcgpu.so")

_synth = None
_gpu = None


class HevcGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hevcgpu error {code}: {msg}")
        self.code = code


# --------------------------------------------------------------------------- synth

def synth_lib():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_SO):
            from . import build
            build.build_synth()
        lib = C.CDLL(SYNTH_SO)
        lib.hevcsynth_default_cfg.argtypes = [C.POINTER(SynthCfg), C.c_int32, C.c_int32, C.c_uint64]
        lib.hevcsynth_default_cfg.restype = None
        lib.hevcsynth_picture.argtypes = [C.POINTER(SynthCfg)]
        lib.hevcsynth_picture.restype = C.POINTER(SynthPicture)
        lib.hevcsynth_picture_free.argtypes = [C.POINTER(SynthPicture)]
        lib.hevcsynth_picture_free.restype = None
        lib.hevcsynth_content.argtypes = [C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_uint8)]
        lib.hevcsynth_content.restype = C.c_int
        lib.hevcsynth_blocks.argtypes = [C.c_int32, C.c_uint64, C.c_int32, C.c_int32, C.POINTER(TU),
                                         C.POINTER(C.c_int16), C.POINTER(C.c_uint8)]
        lib.hevcsynth_blocks.restype = C.c_int64
        lib.hevcsynth_scaling.argtypes = [C.c_uint64, C.POINTER(Scaling)]
        lib.hevcsynth_scaling.restype = C.c_int
        lib.hevcsynth_bs_histogram.argtypes = [C.POINTER(PictureSyntax), C.POINTER(C.c_int64)]
        lib.hevcsynth_bs_histogram.restype = C.c_int
        _synth = lib
    return _synth


def default_cfg(width, height, seed, **kw):
    cfg = SynthCfg()
    synth_lib().hevcsynth_default_cfg(C.byref(cfg), width, height, seed)
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


class Picture:
    """One picture of generated syntax (owns the generator's arrays until freed)."""

    def __init__(self, cfg):
        self._p = synth_lib().hevcsynth_picture(C.byref(cfg))
        if not self._p:
            raise ValueError("hevcsynth_picture: bad configuration")
        self.cfg = cfg

    @property
    def syn(self):
        return self._p.contents.syn

    @property
    def ptr(self):
        return self._p

    @property
    def syn_ptr(self):
        return C.pointer(self._p.contents.syn)

    @property
    def width(self):
        return self.syn.params.width

    @property
    def height(self):
        return self.syn.params.height

    def tus(self):
        n = self.syn.num_tus
        return np.ctypeslib.as_array(C.cast(self.syn.tus, C.POINTER(C.c_uint8)), (n * 16,)).copy() if n else None

    def counts(self):
        s = self.syn
        return {"tus": s.num_tus, "coeffs": s.num_coeffs, "pus": s.num_pus, "wp": s.num_wp,
                "cus": self._p.contents.num_cus}

    def bs_histogram(self):
        out = (C.c_int64 * 3)()
        synth_lib().hevcsynth_bs_histogram(self.syn_ptr, out)
        return list(out)

    # the large record arrays: (field, bytes), in the order and 256-byte alignment of the
    # device buffer that job preparation uploads them into
    def _large_arrays(self):
        s = self.syn
        grid = (s.params.width // 4) * (s.params.height // 4) * 4 if s.blk else 0
        return [("pus", 20 * s.num_pus), ("blk", grid), ("tus", 16 * s.num_tus), ("coeffs", 2 * s.num_coeffs)]

    def pin(self):
        """Moves the large record arrays (PUs, 4x4 grid, TUs, coefficient levels) into one
        block of page-locked memory from hevcgpu_host_alloc, laid out as the device buffer
        they go to (each at a 256-byte aligned offset, in that order), as a recorder that
        writes its records there would: the library uploads them from there in one copy, with
        no staging.  The generator's own arrays are put back before they are freed."""
        if getattr(self, "_pinned", None):
            return self
        lib = gpu_lib()
        s = self.syn
        layout, end = [], 0
        for field, nbytes in self._large_arrays():
            if nbytes <= 0 or not getattr(s, field):
                continue
            off = (end + 255) // 256 * 256
            layout.append((field, nbytes, off))
            end = off + nbytes
        if not layout:
            return self
        block = C.c_void_p()
        _check(lib.hevcgpu_host_alloc(end, C.byref(block)))
        moved = []
        for field, nbytes, off in layout:
            src = getattr(s, field)
            dst = block.value + off
            C.memmove(dst, C.cast(src, C.c_void_p), nbytes)
            moved.append((field, C.cast(src, C.c_void_p).value, type(src)))
            setattr(s, field, C.cast(C.c_void_p(dst), type(src)))
        self._pinned = (block, moved)
        return self

    def _unpin(self):
        pinned = getattr(self, "_pinned", None)
        if pinned:
            block, moved = pinned
            for field, orig, ptype in moved:
                setattr(self.syn, field, C.cast(C.c_void_p(orig), ptype))
            gpu_lib().hevcgpu_host_free(block)
        self._pinned = None

    def close(self):
        if self._p:
            self._unpin()
            synth_lib().hevcsynth_picture_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def content(width, height, seed):
    out = np.empty(i420_size(width, height), np.uint8)
    if synth_lib().hevcsynth_content(width, height, seed, as_ptr(out, C.c_uint8)) != 0:
        raise ValueError("hevcsynth_content: bad size")
    return out


def blocks(num_tus, seed, qp_min=22, qp_max=37):
    """Independent residual blocks: (tus array of TU, coeffs int16, pred uint8)."""
    lib = synth_lib()
    n = lib.hevcsynth_blocks(num_tus, seed, qp_min, qp_max, None, None, None)
    if n < 0:
        raise ValueError("hevcsynth_blocks: bad arguments")
    tus = (TU * max(1, num_tus))()
    coeffs = np.zeros(max(1, n), np.int16)
    pred = np.zeros(max(1, n), np.uint8)
    lib.hevcsynth_blocks(num_tus, seed, qp_min, qp_max, tus, as_ptr(coeffs, C.c_int16), as_ptr(pred, C.c_uint8))
    return tus, num_tus, coeffs, pred


def scaling(seed):
    """Scaling lists (hevc_scaling_t) drawn by the generator from seed."""
    sl = Scaling()
    if synth_lib().hevcsynth_scaling(seed, C.byref(sl)) != 0:
        raise ValueError("hevcsynth_scaling failed")
    return sl


# --------------------------------------------------------------------------- GPU library

def gpu_lib():
    """Load libhevcgpu.so; raises if it is missing (there is no fallback)."""
    global _gpu
    if _gpu is None:
        if not os.path.exists(GPU_SO):
            raise HevcGpuError(abi.HEVCGPU_ECUDA, f"{GPU_SO} is not built (run __graft_entry__.build())")
        lib = C.CDLL(GPU_SO)
        P = C.c_void_p
        u8p = C.POINTER(C.c_uint8)
        sig = {
            "hevcgpu_abi_version": ([], C.c_int),
            "hevcgpu_last_error": ([], C.c_char_p),
            "hevcgpu_create": ([C.c_int, C.POINTER(P)], C.c_int),
            "hevcgpu_destroy": ([P], None),
            "hevcgpu_sync": ([P], C.c_int),
            "hevcgpu_residual_blocks": ([P, C.POINTER(TU), C.c_int32, C.POINTER(C.c_int16), C.c_uint64, u8p, u8p],
                                        C.c_int),
            "hevcgpu_residual_blocks_scaled": ([P, C.POINTER(Scaling), C.POINTER(TU), C.c_int32,
                                                C.POINTER(C.c_int16), C.c_uint64, u8p, u8p], C.c_int),
            "hevcgpu_inter_pred": ([P, C.POINTER(PicParams), C.POINTER(PU), C.c_int32, C.POINTER(WP), C.c_int32,
                                    C.POINTER(u8p), C.c_int32, u8p], C.c_int),
            "hevcgpu_loop_filter": ([P, C.POINTER(PictureSyntax), u8p, u8p, C.c_int, C.c_int], C.c_int),
            "hevcgpu_intra_recon": ([P, C.POINTER(PictureSyntax), u8p, u8p], C.c_int),
            "hevcgpu_reconstruct_picture": ([P, C.POINTER(PictureSyntax), C.POINTER(u8p), C.c_int32, u8p], C.c_int),
            "hevcgpu_set_budget": ([P, C.c_uint64], C.c_int),
            "hevcgpu_bytes_in_use": ([P], C.c_uint64),
            "hevcgpu_stream_open": ([P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(P)], C.c_int),
            "hevcgpu_stream_close": ([P], None),
            "hevcgpu_slot_upload": ([P, C.c_int32, u8p], C.c_int),
            "hevcgpu_slot_download": ([P, C.c_int32, u8p], C.c_int),
            "hevcgpu_slot_download_frame": ([P, C.c_int32, C.POINTER(abi.Crop), C.POINTER(C.c_uint16), C.c_int32,
                                             C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), C.c_int32], C.c_int),
            "hevcgpu_slot_checksum": ([P, C.c_int32, C.POINTER(abi.Crop), C.POINTER(C.c_uint32)], C.c_int),
            "hevcgpu_intra_schedule": ([P, C.POINTER(abi.IntraSchedule)], C.c_int),
            "hevcgpu_mc_strips": ([P, C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_int32),
                                   C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_int32)], C.c_int),
            "hevcgpu_slot_device_ptr": ([P, C.c_int32, C.POINTER(P), C.POINTER(P), C.POINTER(P),
                                         C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
            "hevcgpu_job_prepare": ([P, C.POINTER(PictureSyntax), C.POINTER(P)], C.c_int),
            "hevcgpu_job_wait_uploaded": ([P], C.c_int),
            "hevcgpu_job_plant_unmet_wait": ([P], C.c_int),
            "hevcgpu_job_free": ([P], None),
            "hevcgpu_job_upload_bytes": ([P], C.c_uint64),
            "hevcgpu_host_alloc": ([C.c_size_t, C.POINTER(P)], C.c_int),
            "hevcgpu_host_free": ([P], C.c_int),
            "hevcgpu_job_launch": ([P, C.c_int32], C.c_int),
            "hevcgpu_batch_launch": ([C.POINTER(P), C.POINTER(C.c_int32), C.c_int32], C.c_int),
            "hevcgpu_stream_sync": ([P], C.c_int),
            "hevcgpu_jobs_prepare": ([C.POINTER(P), C.POINTER(P), C.c_int32, C.POINTER(P)], C.c_int),
            "hevcgpu_jobs_prepare_async": ([C.POINTER(P), C.POINTER(P), C.c_int32, C.POINTER(P)], C.c_int),
            "hevcgpu_lane_open": ([P, C.POINTER(P)], C.c_int),
            "hevcgpu_lane_close": ([P], None),
            "hevcgpu_lane_batch_launch": ([P, C.POINTER(P), C.POINTER(C.c_int32), C.c_int32], C.c_int),
            "hevcgpu_lane_sync": ([P], C.c_int),
            "hevcgpu_lane_cuda_stream": ([P], P),
            "hevcgpu_lane_copy_stream": ([P], P),
            "hevcgpu_lane_slots_download": ([P, C.POINTER(P), C.POINTER(C.c_int32), C.c_int32, C.POINTER(P)],
                                            C.c_int),
            "hevcgpu_lane_slots_download_async": ([P, C.POINTER(P), C.POINTER(C.c_int32), C.c_int32,
                                                   C.POINTER(P), C.POINTER(C.c_uint64)], C.c_int),
            "hevcgpu_lane_wait": ([P, C.c_uint64], C.c_int),
            "hevcgpu_slots_download": ([C.POINTER(P), C.POINTER(C.c_int32), C.c_int32, C.POINTER(P)], C.c_int),
            "hevcgpu_cuda_stream": ([P], P),
            "hevcgpu_launch_count": ([P], C.c_uint64),
            "hevcgpu_picture_decode": ([P, C.POINTER(PictureSyntax), C.c_int32], C.c_int),
            "hevcgpu_profile_enable": ([P, C.c_int], C.c_int),
            "hevcgpu_profile_read": ([P, C.POINTER(C.c_double), C.POINTER(C.c_uint64)], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        _gpu = lib
    return _gpu


def _check(code):
    if code < 0:
        msg = gpu_lib().hevcgpu_last_error()
        raise HevcGpuError(code, msg.decode() if msg else "")
    return code


class Context:
    """A CUDA context of the back end on one device (hevcgpu_create)."""

    def __init__(self, device=0):
        self.lib = gpu_lib()
        self._children = weakref.WeakSet()   # streams, lanes and jobs: closed before the context
        h = C.c_void_p()
        _check(self.lib.hevcgpu_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            kids = list(self._children)
            for k in kids:
                if isinstance(k, Job):
                    k.free()
            for k in kids:
                if isinstance(k, (Stream, Lane)):
                    k.close()
            self.lib.hevcgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        _check(self.lib.hevcgpu_sync(self.h))

    @property
    def launches(self):
        return int(self.lib.hevcgpu_launch_count(self.h))

    @property
    def cuda_stream(self):
        return self.lib.hevcgpu_cuda_stream(self.h)

    STAGES = ("motion_grid", "mc", "residual", "intra", "deblock_v", "deblock_h", "sao")

    def profile(self, enable=True):
        _check(self.lib.hevcgpu_profile_enable(self.h, int(enable)))

    def profile_read(self):
        ms = (C.c_double * 7)()
        n = (C.c_uint64 * 7)()
        _check(self.lib.hevcgpu_profile_read(self.h, ms, n))
        return {s: (ms[i], int(n[i])) for i, s in enumerate(self.STAGES)}

    # ---- stages on host memory
    def residual_blocks(self, tus, num_tus, coeffs, pred, scaling=None):
        """scaling: an abi.Scaling (scaling_list_enabled_flag = 1) or None (flat)."""
        out = np.empty_like(pred)
        _check(self.lib.hevcgpu_residual_blocks_scaled(
            self.h, C.byref(scaling) if scaling is not None else None, tus, num_tus, as_ptr(coeffs, C.c_int16),
            coeffs.size, as_ptr(pred, C.c_uint8), as_ptr(out, C.c_uint8)))
        return out

    def inter_pred(self, pic, refs):
        p = pic.syn.params
        out = np.zeros(i420_size(p.width, p.height), np.uint8)
        _check(self.lib.hevcgpu_inter_pred(self.h, C.byref(p), pic.syn.pus, pic.syn.num_pus, pic.syn.wp,
                                           pic.syn.num_wp, ptr_array(refs), len(refs), as_ptr(out, C.c_uint8)))
        return out

    def loop_filter(self, pic, inp, do_deblock=True, do_sao=True):
        out = np.empty_like(inp)
        _check(self.lib.hevcgpu_loop_filter(self.h, pic.syn_ptr, as_ptr(inp, C.c_uint8), as_ptr(out, C.c_uint8),
                                            int(do_deblock), int(do_sao)))
        return out

    def intra_recon(self, pic, inp):
        out = np.empty_like(inp)
        _check(self.lib.hevcgpu_intra_recon(self.h, pic.syn_ptr, as_ptr(inp, C.c_uint8), as_ptr(out, C.c_uint8)))
        return out

    def reconstruct_picture(self, pic, refs):
        p = pic.syn.params
        out = np.zeros(i420_size(p.width, p.height), np.uint8)
        _check(self.lib.hevcgpu_reconstruct_picture(self.h, pic.syn_ptr, ptr_array(refs), len(refs),
                                                    as_ptr(out, C.c_uint8)))
        return out

    # ---- DPB / picture pipeline
    def set_budget(self, nbytes):
        _check(self.lib.hevcgpu_set_budget(self.h, nbytes))

    def bytes_in_use(self):
        return int(self.lib.hevcgpu_bytes_in_use(self.h))

    def open_stream(self, width, height, slots):
        return Stream(self, width, height, slots)


class Stream:
    """A decode stream: DPB slots in HBM (hevcgpu_stream_open)."""

    def __init__(self, ctx, width, height, slots):
        self.ctx = ctx
        self.lib = ctx.lib
        self.width, self.height, self.slots = width, height, slots
        h = C.c_void_p()
        _check(self.lib.hevcgpu_stream_open(ctx.h, width, height, 8, slots, C.byref(h)))
        self.h = h
        ctx._children.add(self)

    def close(self):
        if self.h and self.ctx.h:
            self.lib.hevcgpu_stream_close(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, slot, i420):
        _check(self.lib.hevcgpu_slot_upload(self.h, slot, as_ptr(i420, C.c_uint8)))

    def download(self, slot, out=None):
        if out is None:
            out = np.empty(i420_size(self.width, self.height), np.uint8)
        _check(self.lib.hevcgpu_slot_download(self.h, slot, as_ptr(out, C.c_uint8)))
        return out

    def download_frame(self, slot, crop=None, stride_y=None, stride_c=None):
        """The slot as hevc_decoder_get_frame gives a picture (hevcgpu_slot_download_frame):
        (y, cb, cr) uint16 planes inside the conformance window crop = (left, right, top,
        bottom) in luma samples, each a view of width x height samples of rows of the stride."""
        left, right, top, bottom = crop or (0, 0, 0, 0)
        w, h = self.width - left - right, self.height - top - bottom
        sy, sc = stride_y or w, stride_c or w // 2
        bufs = [np.zeros((h, sy), np.uint16), np.zeros((h // 2, sc), np.uint16), np.zeros((h // 2, sc), np.uint16)]
        c = abi.Crop(left, right, top, bottom)
        _check(self.lib.hevcgpu_slot_download_frame(self.h, slot, C.byref(c), as_ptr(bufs[0], C.c_uint16), sy,
                                                    as_ptr(bufs[1], C.c_uint16), as_ptr(bufs[2], C.c_uint16), sc))
        return bufs[0][:, :w], bufs[1][:, :w // 2], bufs[2][:, :w // 2]

    def checksum(self, slot, crop=None):
        """(Y, Cb, Cr) checksums of the slot's frame (hevcgpu_slot_checksum: the H.265
        picture hash SEI checksum over the conformance window crop = (left, right, top,
        bottom)), computed on the device."""
        left, right, top, bottom = crop or (0, 0, 0, 0)
        c = abi.Crop(left, right, top, bottom)
        out = (C.c_uint32 * 3)()
        _check(self.lib.hevcgpu_slot_checksum(self.h, slot, C.byref(c), out))
        return tuple(out)

    def prepare(self, pic):
        return Job(self, pic)

    def decode(self, pic, dst_slot):
        _check(self.lib.hevcgpu_picture_decode(self.h, pic.syn_ptr, dst_slot))

    def sync(self):
        _check(self.lib.hevcgpu_stream_sync(self.h))


class Job:
    """A prepared picture (records uploaded once; hevcgpu_job_prepare)."""

    def __init__(self, stream, pic, handle=None):
        self.stream = stream
        self.lib = stream.lib
        if handle is None:
            handle = C.c_void_p()
            _check(self.lib.hevcgpu_job_prepare(stream.h, pic.syn_ptr, C.byref(handle)))
        self.h = handle
        stream.ctx._children.add(self)

    def plant_unmet_wait(self):
        """Test hook: the job's next launch times out in its intra stage (HEVCGPU_ETIMEOUT
        at the next sync); hevcgpu_job_plant_unmet_wait."""
        _check(self.lib.hevcgpu_job_plant_unmet_wait(self.h))

    def wait_uploaded(self):
        """Returns once the copies of the picture's page-locked record arrays have read them."""
        _check(self.lib.hevcgpu_job_wait_uploaded(self.h))

    def launch(self, dst_slot):
        _check(self.lib.hevcgpu_job_launch(self.h, dst_slot))

    @property
    def upload_bytes(self):
        return int(self.lib.hevcgpu_job_upload_bytes(self.h))

    def free(self):
        if self.h and self.stream.h and self.stream.ctx.h:
            self.lib.hevcgpu_job_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def batch_launch(jobs, dst_slots):
    lib = gpu_lib()
    n = len(jobs)
    arr = (C.c_void_p * n)(*[j.h for j in jobs])
    slots = (C.c_int32 * n)(*dst_slots)
    _check(lib.hevcgpu_batch_launch(arr, slots, n))


class Lane:
    """A launch queue of a context that runs side by side with the others
    (hevcgpu_lane_open): batches on different lanes overlap on the device."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        _check(self.lib.hevcgpu_lane_open(ctx.h, C.byref(h)))
        self.h = h
        ctx._children.add(self)

    def batch_launch(self, jobs, dst_slots):
        n = len(jobs)
        arr = (C.c_void_p * n)(*[j.h for j in jobs])
        slots = (C.c_int32 * n)(*dst_slots)
        _check(self.lib.hevcgpu_lane_batch_launch(self.h, arr, slots, n))

    def sync(self):
        _check(self.lib.hevcgpu_lane_sync(self.h))

    def download_batch(self, streams, slots, outs):
        """Slots of streams into host buffers, the copies ordered after this lane's batches."""
        n = len(streams)
        sts = (C.c_void_p * n)(*[st.h for st in streams])
        sl = (C.c_int32 * n)(*slots)
        ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        _check(self.lib.hevcgpu_lane_slots_download(self.h, sts, sl, n, ptrs))
        return outs

    def download_batch_async(self, streams, slots, outs):
        """The same copies into page-locked host buffers, queued without waiting; returns
        the ticket to pass to wait() before reading the buffers."""
        n = len(streams)
        sts = (C.c_void_p * n)(*[st.h for st in streams])
        sl = (C.c_int32 * n)(*slots)
        ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        ticket = C.c_uint64()
        _check(self.lib.hevcgpu_lane_slots_download_async(self.h, sts, sl, n, ptrs, C.byref(ticket)))
        return ticket.value

    def wait(self, ticket):
        """Returns once the download with this ticket has landed."""
        _check(self.lib.hevcgpu_lane_wait(self.h, ticket))

    @property
    def cuda_stream(self):
        return self.lib.hevcgpu_lane_cuda_stream(self.h)

    @property
    def copy_stream(self):
        """CUDA stream of the lane's asynchronous downloads (hevcgpu_lane_copy_stream)."""
        return self.lib.hevcgpu_lane_copy_stream(self.h)

    def close(self):
        if self.h and self.ctx.h:
            self.lib.hevcgpu_lane_close(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def intra_schedule(pic):
    """The intra schedule the back end builds for a picture (hevcgpu_intra_schedule; host
    work only): a dict of numpy copies of its arrays."""
    lib = gpu_lib()
    out = abi.IntraSchedule()
    _check(lib.hevcgpu_intra_schedule(C.cast(pic.syn_ptr, C.c_void_p), C.byref(out)))

    def arr(ptr, n, dt):
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt) if n > 0 else np.zeros(0, dt)
    return {"ctu_addr": arr(out.ctu_addr, out.n_ctu, np.int64), "ctu_first": arr(out.ctu_first, out.n_ctu + 1, np.int64),
            "task_tu": arr(out.task_tu, out.n_task, np.int64), "task_deps": arr(out.task_deps, out.n_task, np.uint32),
            "deps": arr(out.deps, out.n_dep, np.uint32), "task_flags": arr(out.task_flags, out.n_task, np.uint8),
            "ctu_watch": arr(out.ctu_watch, out.n_ctu, np.uint32), "watch": arr(out.watch, out.n_watch, np.int64)}


def mc_strips(pic):
    """The MC strip lists the back end builds for a picture (hevcgpu_mc_strips; host work
    only): (luma items, chroma items) as numpy copies."""
    lib = gpu_lib()
    lp, cp = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    nl, nc = C.c_int32(0), C.c_int32(0)
    _check(lib.hevcgpu_mc_strips(C.cast(pic.syn_ptr, C.c_void_p), C.byref(lp), C.byref(nl), C.byref(cp), C.byref(nc)))

    def arr(ptr, n):
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n > 0 else np.zeros(0, np.uint32)
    return arr(lp, nl.value), arr(cp, nc.value)


def prepare_batch(streams, pics, wait_uploads=True):
    """Jobs for pics[i] on streams[i], built on the context's host workers
    (hevcgpu_jobs_prepare).  wait_uploads=False: hevcgpu_jobs_prepare_async, which returns
    with the copies of page-locked record arrays still in flight (Job.wait_uploaded before
    writing into them)."""
    lib = gpu_lib()
    n = len(pics)
    sts = (C.c_void_p * n)(*[st.h for st in streams])
    syns = (C.c_void_p * n)(*[C.cast(p.syn_ptr, C.c_void_p) for p in pics])
    out = (C.c_void_p * n)()
    f = lib.hevcgpu_jobs_prepare if wait_uploads else lib.hevcgpu_jobs_prepare_async
    _check(f(sts, syns, n, out))
    return [Job(st, None, C.c_void_p(h)) for st, h in zip(streams, out)]


def download_batch(streams, slots, outs=None):
    """Slot slots[i] of streams[i] into I420 host buffers (hevcgpu_slots_download)."""
    lib = gpu_lib()
    n = len(streams)
    if outs is None:
        outs = [np.empty(i420_size(st.width, st.height), np.uint8) for st in streams]
    sts = (C.c_void_p * n)(*[st.h for st in streams])
    sl = (C.c_int32 * n)(*slots)
    ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
    _check(lib.hevcgpu_slots_download(sts, sl, n, ptrs))
    return outs
