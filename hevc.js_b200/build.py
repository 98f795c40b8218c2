"""In-tree build of the native libraries of the package.

  libhevcsynth.so  host: seeded workload generator (csrc/synth.cpp)
  libhevcgpu.so    the CUDA back end for sm_100a (csrc/hevcgpu.cu + kernels) with the
                   C ABI of include/hevcgpu.h

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
GPU_SO = os.path.join(PKG, "libhevcgpu.so")

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


def build_all(force=False):
    build_synth(force)
    build_gpu(force)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(build_gpu(force=True, verbose_ptxas=True))
    else:
        build_all(force="--force" in sys.argv)
