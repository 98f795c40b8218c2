"""hevcgpu_residual_blocks_static — residual blocks on caller-owned device buffers with
no allocation inside the call — gives the same bytes as hevcgpu_residual_blocks.

Collected after the other test files (file name) so that it runs both after their GPU tests
(those marked `last` aside) and, when selected alone, in a fresh process where its first
call does the per-device set-up."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_fn(hb):
    from hevc_b200 import abi
    lib = hb.gpu_lib()
    f = lib.hevcgpu_residual_blocks_static
    f.argtypes = [C.c_void_p, C.POINTER(abi.TU), C.c_int32, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return lib, f


def _run_static(hb, ctx, f, tus, n, coeffs, pred):
    import torch
    dev = torch.device("cuda", 0)
    d_coeffs = torch.from_numpy(coeffs).to(dev)
    d_pred = torch.from_numpy(pred).to(dev)
    d_out = torch.zeros(pred.size, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    rc = f(ctx.h, tus, n, d_coeffs.data_ptr(), coeffs.size, d_pred.data_ptr(), d_out.data_ptr())
    assert rc == 0, hb.gpu_lib().hevcgpu_last_error()
    return d_out.cpu().numpy()


@pytest.mark.parametrize("num_tus,seed", [(3000, 71), (257, 72)])
def test_static_matches_residual_blocks_twice(hb, gpu_ctx, num_tus, seed):
    lib, f = _static_fn(hb)
    tus, n, coeffs, pred = hb.blocks(num_tus, seed)
    want = gpu_ctx.residual_blocks(tus, n, coeffs, pred)
    first = _run_static(hb, gpu_ctx, f, tus, n, coeffs, pred)
    second = _run_static(hb, gpu_ctx, f, tus, n, coeffs, pred)
    assert np.array_equal(first, want)
    assert np.array_equal(second, want)


def test_static_two_inputs_in_a_row(hb, gpu_ctx):
    lib, f = _static_fn(hb)
    a = hb.blocks(1500, 73)
    b = hb.blocks(900, 74, qp_min=40, qp_max=51)
    got_a = _run_static(hb, gpu_ctx, f, *a)
    got_b = _run_static(hb, gpu_ctx, f, *b)
    assert np.array_equal(got_a, gpu_ctx.residual_blocks(*a))
    assert np.array_equal(got_b, gpu_ctx.residual_blocks(*b))


def test_static_rejects_more_blocks_than_its_scratch(hb, gpu_ctx):
    from hevc_b200 import abi
    lib, f = _static_fn(hb)
    limit = 65536
    tus = (abi.TU * 1)()
    rc = f(gpu_ctx.h, tus, limit + 1, None, 0, None, None)
    assert rc == abi.HEVCGPU_EINVAL
    assert b"at most 65536" in lib.hevcgpu_last_error()


def test_static_rejects_host_buffers(hb, gpu_ctx):
    from hevc_b200 import abi
    lib, f = _static_fn(hb)
    tus, n, coeffs, pred = hb.blocks(16, 75)
    out = np.zeros_like(pred)
    rc = f(gpu_ctx.h, tus, n, coeffs.ctypes.data, coeffs.size, pred.ctypes.data, out.ctypes.data)
    assert rc == abi.HEVCGPU_EINVAL


def test_static_block_ending_at_the_pool_end(hb, gpu_ctx):
    """The last block's levels end exactly at num_coeffs (accepted, same bytes); one level
    fewer in the pool is refused."""
    import torch
    from hevc_b200 import abi
    lib, f = _static_fn(hb)
    tus, n, coeffs, pred = hb.blocks(300, 76)
    ends = [tus[i].coeff_offset + (1 << (2 * tus[i].log2_size)) for i in range(n)]
    assert max(ends) == coeffs.size
    assert np.array_equal(_run_static(hb, gpu_ctx, f, tus, n, coeffs, pred), gpu_ctx.residual_blocks(tus, n, coeffs, pred))
    dev = torch.device("cuda", 0)
    d_coeffs = torch.from_numpy(coeffs).to(dev)
    d_pred = torch.from_numpy(pred).to(dev)
    d_out = torch.zeros(pred.size, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    rc = f(gpu_ctx.h, tus, n, d_coeffs.data_ptr(), coeffs.size - 1, d_pred.data_ptr(), d_out.data_ptr())
    assert rc == abi.HEVCGPU_EINVAL


def test_static_rejects_unaligned_device_buffers(hb, gpu_ctx):
    import torch
    from hevc_b200 import abi
    lib, f = _static_fn(hb)
    tus, n, coeffs, pred = hb.blocks(16, 77)
    dev = torch.device("cuda", 0)
    d_coeffs = torch.zeros(coeffs.size + 8, dtype=torch.int16, device=dev)
    d_pred = torch.from_numpy(pred).to(dev)
    d_out = torch.zeros(pred.size, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    rc = f(gpu_ctx.h, tus, n, d_coeffs.data_ptr() + 2, coeffs.size, d_pred.data_ptr(), d_out.data_ptr())
    assert rc == abi.HEVCGPU_EINVAL
    assert b"aligned" in lib.hevcgpu_last_error()
