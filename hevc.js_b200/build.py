"""In-tree build of the native libraries of the package.

  libhevcsynth.so  host: seeded workload generator (csrc/synth.cpp)
  libhevcgpu.so    the CUDA back end for sm_100a (csrc/hevcgpu.cu + kernels) with the
                   C ABI of include/hevcgpu.h
  libhevcdec_gpu.so  the hevc.js decoder C API (include/hevc_api_gpu.h): the reference's
                   host parser compiled from its sources (HEVC_REF_DIR, or a checkout beside
                   this repository) with the recording hooks of dropin/, over libhevcgpu.so;
                   built only where the reference tree is present (the built library travels)

Both are written next to this file so that they travel with the source tree.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SYNTH_SO = os.path.join(PKG, "libhevcsynth.so")
BITGEN_SO = os.path.join(PKG, "libhevcbitgen.so")
GPU_SO = os.path.join(PKG, "libhevcgpu.so")
DROPIN_SO = os.path.join(PKG, "libhevcdec_gpu.so")
DROPIN_CLI = os.path.join(PKG, "dropin", "_build", "hevc-decode")

GPU_SOURCES = ["hevcgpu.cu"]
GPU_DEPS = ["hevcgpu.cu", "kernels.cuh", "mc.cuh", "intra.cuh", "device_common.cuh", "../../include/hevcgpu.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd)}")
    return r.stdout + r.stderr


def build_synth(force=False):
    src = os.path.join(CSRC, "synth.cpp")
    deps = [src, os.path.join(CSRC, "synth.h"), os.path.join(ROOT, "include", "hevcgpu.h")]
    if force or _newer(SYNTH_SO, deps):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-o", SYNTH_SO, src])
    return SYNTH_SO


def build_gpu(force=False, verbose_ptxas=False):
    srcs = [os.path.join(CSRC, s) for s in GPU_SOURCES]
    deps = [os.path.join(CSRC, d) for d in GPU_DEPS]
    if force or _newer(GPU_SO, deps):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               "-I", os.path.join(ROOT, "include"), "-o", GPU_SO, *srcs, "-lcudart"]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        out = _run(cmd)
        if verbose_ptxas:
            return out
    return GPU_SO


def ref_dir():
    return os.environ.get("HEVC_REF_DIR", os.path.join(os.path.dirname(ROOT), "reference"))


def build_dropin(force=False):
    """The drop-in decoder library and the reference's CLI over it (dropin/Makefile)."""
    ref = ref_dir()
    if not os.path.isdir(os.path.join(ref, "src")):
        return None
    cmd = ["make", "-s", "-C", os.path.join(PKG, "dropin"), f"REF_DIR={ref}", "-j8"]
    if force:
        cmd.insert(1, "-B")
    _run(cmd)
    return DROPIN_SO


def build_bitgen(force=False):
    """The random-syntax bitstream generator (host code, csrc/bitgen.cpp)."""
    src = os.path.join(CSRC, "bitgen.cpp")
    deps = [src, os.path.join(CSRC, "bitgen.h"), os.path.join(ROOT, "include", "hevcgpu.h")]
    if force or _newer(BITGEN_SO, deps):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I", os.path.join(ROOT, "include"),
              "-o", BITGEN_SO, src])
    return BITGEN_SO


def build_all(force=False):
    build_synth(force)
    build_bitgen(force)
    build_gpu(force)
    build_dropin(force)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(build_gpu(force=True, verbose_ptxas=True))
    else:
        build_all(force="--force" in sys.argv)
