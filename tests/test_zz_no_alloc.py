"""The allocation-free CC pair entry point against the ordinary one, through the C ABI.

fw_cc_value_derivative_pair_noalloc serves callers that cannot allocate device memory (hosts
whose own pool allocator owns the GPU, plug-ins handed only their buffers, real-time pipelines
with pre-planned memory): they pass every input and output, and the kernel's scratch is a static
array inside the library. This file runs after every other test (pytest collects it
last) and also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from cases import CASES, image
from fastwarp_b200 import CudaBackend, make_grid
from fastwarp_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["awkward_aligned", "awkward_oblique"])
def test_the_allocation_free_cc_pair_matches_the_ordinary_entry_point(name):
    import torch

    case = CASES[name]
    g = make_grid(case["size"], case["spacing"], case["origin"], case["direction"])
    og = O.make_grid(case["size"], case["spacing"], case["origin"], case["direction"])
    r = case["radius"]
    fimg, mimg = image(case), image(case, seed_offset=5)
    lib = N.lib()
    with CudaBackend(0) as b:
        fi = b.upload_image(g, fimg.astype(np.float32))
        mi = b.upload_image(g, mimg.astype(np.float32))
        (v1, d1), (v2, d2) = b.cc_value_derivative_pair(fi, mi, r)
        want1, want2 = b.download_field(d1), b.download_field(d2)
        # outputs owned by the caller: two fields and a 3-double result on the device
        out1, out2 = b.zero_field(g), b.zero_field(g)
        ps1, ps2 = C.c_int64(), C.c_int64()
        p1 = lib.fw_field_device_ptr(out1.handle, C.byref(ps1))
        p2 = lib.fw_field_device_ptr(out2.handle, C.byref(ps2))
        assert ps1.value == ps2.value
        result = torch.zeros(3, dtype=torch.float64, device="cuda:0")
        stream = lib.fw_ctx_stream(b.ctx)
        for call in range(2):  # two calls in a row share (and must clear) the static scratch
            N.check(lib.fw_cc_value_derivative_pair_noalloc(
                C.byref(g), C.c_void_p(lib.fw_image_device_ptr(fi.handle)),
                C.c_void_p(lib.fw_image_device_ptr(mi.handle)), C.c_int32(r), C.c_void_p(p1),
                C.c_void_p(p2), ps1, C.c_void_p(result.data_ptr()), C.c_void_p(stream)))
            b.synchronize()
            value, n1, n2 = result.cpu().tolist()
            got1, got2 = b.download_field(out1), b.download_field(out2)
            assert abs(value - v1) <= 1e-5 * abs(v1), (call, value, v1)
            assert np.abs(got1 - want1).max() <= 1e-4 * np.abs(want1).max()
            assert np.abs(got2 - want2).max() <= 1e-4 * np.abs(want2).max()
            assert abs(np.sqrt(n1) - np.sqrt((want1 ** 2).sum())) <= 1e-5 * np.sqrt((want1 ** 2).sum())
            assert abs(np.sqrt(n2) - np.sqrt((want2 ** 2).sum())) <= 1e-5 * np.sqrt((want2 ** 2).sum())
        # and both agree with the f64 oracle
        (w1, _), _ = O.cc_pair(og, fimg, mimg, r)
        assert abs(value - w1) <= 1e-5 * abs(w1)


def test_the_allocation_free_cc_pair_rejects_grids_beyond_its_scratch():
    lib = N.lib()
    g = make_grid((4096, 4096, 8))  # 128 x 512 tiles > FW_NOALLOC_MAX_BLOCKS
    rc = lib.fw_cc_value_derivative_pair_noalloc(
        C.byref(g), C.c_void_p(16), C.c_void_p(16), C.c_int32(2), C.c_void_p(16),
        C.c_void_p(16), C.c_int64(4096 * 4096 * 8), C.c_void_p(16), None)
    assert rc == N.FW_ERR_INVALID
    assert b"static scratch" in lib.fw_last_error()
