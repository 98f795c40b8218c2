"""The C-ABI library: it loads, exports every declared entry point, its record layouts
match the header, and it refuses to run without a CUDA device (no CPU fallback)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hevcgpu.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(hevcgpu_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib(hb):
    from hevc_b200 import build
    build.build_gpu()
    return C.CDLL(hb.GPU_SO)


def test_header_declares_entry_points():
    names = declared()
    assert "hevcgpu_create" in names and "hevcgpu_reconstruct_picture" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_record_layouts_match_header(hb, tmp_path):
    hb.abi.check_layouts()
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "hevcgpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(hevc_tu_t), sizeof(hevc_pu_t), sizeof(hevc_wp_t),
         sizeof(hevc_sao_t), sizeof(hevc_slice_t), sizeof(hevc_pic_params_t), sizeof(hevc_picture_syntax_t),
         sizeof(hevc_intra_schedule_t));
  printf("%zu %zu %zu %zu %zu\\n", offsetof(hevc_picture_syntax_t, tus), offsetof(hevc_picture_syntax_t, coeffs),
         offsetof(hevc_picture_syntax_t, blk), offsetof(hevc_picture_syntax_t, slices),
         offsetof(hevc_pic_params_t, ref_slot));
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in out[0].split()]
    offs = [int(x) for x in out[1].split()]
    a = hb.abi
    assert sizes == [C.sizeof(a.TU), C.sizeof(a.PU), C.sizeof(a.WP), C.sizeof(a.SAO), C.sizeof(a.Slice),
                     C.sizeof(a.PicParams), C.sizeof(a.PictureSyntax), C.sizeof(a.IntraSchedule)]
    assert offs == [a.PictureSyntax.tus.offset, a.PictureSyntax.coeffs.offset, a.PictureSyntax.blk.offset,
                    a.PictureSyntax.slices.offset, a.PicParams.ref_slot.offset]


def test_picture_checksum_helper_follows_the_sei_definition():
    """The tests' checksum of a plane (the one hevcgpu_slot_checksum computes on the device)
    against the definition's loop, sample by sample, on a plane with coordinates past 255."""
    import cases
    rng = np.random.default_rng(7)
    plane = rng.integers(0, 256, size=(261, 300), dtype=np.uint8)
    want = 0
    for yy in range(plane.shape[0]):
        for xx in range(plane.shape[1]):
            mask = (xx & 0xFF) ^ (yy & 0xFF) ^ (xx >> 8) ^ (yy >> 8)
            want = (want + ((int(plane[yy, xx]) & 0xFF) ^ mask)) & 0xFFFFFFFF
    assert cases.picture_checksum(plane) == want
    assert cases.picture_checksum(np.zeros((2, 2), np.uint8)) == 0 + 1 + 1 + 0


def test_abi_version(lib):
    lib.hevcgpu_abi_version.restype = C.c_int
    assert lib.hevcgpu_abi_version() == 2


def test_create_fails_loudly_without_gpu(hb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hb.HevcGpuError) as e:
        hb.Context(0)
    assert e.value.code in (hb.abi.HEVCGPU_ECUDA, hb.abi.HEVCGPU_EUNSUPPORTED)


def test_kernels_are_built_for_sm100a(hb):
    from hevc_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert os.path.exists(hb.GPU_SO)
