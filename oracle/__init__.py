"""Checkers for the reconstruction back end — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm load
this.  Two checkers share one calling convention (the records of include/hevcgpu.h):

  port  oracle/_build/liboracle.so  CPU restatement of the reference (hevc_oracle.c);
                                    built from this repository on any machine.
  ref   oracle/_ref/libhevcref.so   privaloops/hevc.js's own functions compiled from its
                                    sources by oracle/Makefile (needs the reference tree
                                    at build time; the built library travels).
"""
import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhevcref.so")
REF_CLI = os.path.join(HERE, "_ref", "hevc-decode")
RECORDER = os.path.join(HERE, "_ref", "hevc-record")
DROPIN_SO = os.path.join(HERE, "_ref", "libhevcdec_oracle.so")
# the reference tree: HEVC_REF_DIR, else a checkout beside this repository
REF_DIR = os.environ.get("HEVC_REF_DIR", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))

_libs = {}


def build(with_ref=None):
    """Build the port always, and the reference harness when its sources are present."""
    targets = ["oracle"]
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(REF_DIR, "src"))
    if with_ref:
        targets += ["ref", "record", "dropin"]
    subprocess.run(["make", "-s", "-C", HERE, f"REF_DIR={REF_DIR}", "-j8", *targets], check=True)


def _bind(lib, prefix, syn_t):
    from importlib import import_module
    abi = import_module("hevc_b200.abi")
    u8p = C.POINTER(C.c_uint8)
    sig = {
        "residual_blocks": ([C.POINTER(abi.TU), C.c_int32, C.POINTER(C.c_int16), u8p, u8p], C.c_int),
        "residual_blocks_scaled": ([C.POINTER(abi.Scaling), C.POINTER(abi.TU), C.c_int32, C.POINTER(C.c_int16),
                                    u8p, u8p], C.c_int),
        "inter_pred": ([C.POINTER(abi.PicParams), C.POINTER(abi.PU), C.c_int32, C.POINTER(abi.WP), C.c_int32,
                        C.POINTER(u8p), C.c_int32, u8p], C.c_int),
        "loop_filter": ([C.POINTER(abi.PictureSyntax), u8p, u8p, C.c_int, C.c_int], C.c_int),
        "intra_recon": ([C.POINTER(abi.PictureSyntax), u8p, u8p], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, prefix + name)
        f.argtypes = args
        f.restype = res
    f = getattr(lib, prefix + "reconstruct_picture")
    f.argtypes = [C.POINTER(syn_t), C.POINTER(u8p), C.c_int32, u8p]
    f.restype = C.c_int
    return lib


def port():
    if "port" not in _libs:
        if not os.path.exists(PORT_SO):
            build(with_ref=False)
        from importlib import import_module
        abi = import_module("hevc_b200.abi")
        _libs["port"] = Checker(_bind(C.CDLL(PORT_SO), "oracle_", abi.PictureSyntax), "port")
    return _libs["port"]


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    if "ref" not in _libs:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        from importlib import import_module
        abi = import_module("hevc_b200.abi")
        _libs["ref"] = Checker(_bind(C.CDLL(REF_SO), "ref_", abi.SynthPicture), "ref")
    return _libs["ref"]


class Checker:
    """Same entry points for the port and the reference harness (numpy in/out)."""

    def __init__(self, lib, kind):
        self.lib = lib
        self.kind = kind
        self.prefix = "oracle_" if kind == "port" else "ref_"

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def residual_blocks(self, tus, num_tus, coeffs, pred, scaling=None):
        import numpy as np
        from hevc_b200.abi import as_ptr
        out = np.empty_like(pred)
        sl = C.byref(scaling) if scaling is not None else None
        rc = self._f("residual_blocks_scaled")(sl, tus, num_tus, as_ptr(coeffs, C.c_int16), as_ptr(pred, C.c_uint8),
                                               as_ptr(out, C.c_uint8))
        assert rc == 0
        return out

    def inter_pred(self, pic, refs):
        import numpy as np
        from hevc_b200.abi import as_ptr, ptr_array, i420_size
        p = pic.syn.params
        out = np.zeros(i420_size(p.width, p.height), np.uint8)
        rc = self._f("inter_pred")(C.byref(p), pic.syn.pus, pic.syn.num_pus, pic.syn.wp, pic.syn.num_wp,
                                   ptr_array(refs), len(refs), as_ptr(out, C.c_uint8))
        assert rc == 0
        return out

    def loop_filter(self, pic, inp, do_deblock=True, do_sao=True):
        import numpy as np
        from hevc_b200.abi import as_ptr
        out = np.empty_like(inp)
        rc = self._f("loop_filter")(pic.syn_ptr, as_ptr(inp, C.c_uint8), as_ptr(out, C.c_uint8), int(do_deblock),
                                    int(do_sao))
        assert rc == 0
        return out

    def intra_recon(self, pic, inp):
        import numpy as np
        from hevc_b200.abi import as_ptr
        out = np.empty_like(inp)
        rc = self._f("intra_recon")(pic.syn_ptr, as_ptr(inp, C.c_uint8), as_ptr(out, C.c_uint8))
        assert rc == 0
        return out

    def reconstruct_picture(self, pic, refs):
        import numpy as np
        from hevc_b200.abi import as_ptr, ptr_array, i420_size
        p = pic.syn.params
        out = np.zeros(i420_size(p.width, p.height), np.uint8)
        arg = pic.syn_ptr if self.kind == "port" else pic.ptr
        rc = self._f("reconstruct_picture")(arg, ptr_array(refs), len(refs), as_ptr(out, C.c_uint8))
        assert rc == 0
        return out
