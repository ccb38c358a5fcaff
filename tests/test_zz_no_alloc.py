"""The allocation-free block map entry point, through the C ABI.

sred_block_map_2d_device_noalloc serves callers that cannot call cudaMalloc
(a host runtime that owns the device allocator, a real-time loop that must
not allocate). It keeps its scratch in a fixed
device array shared by all calls, so this test checks two calls in a row on
different inputs (nothing left over from the first call may leak into the
second) against the regular entry point, sred_block_map_2d_device, with the
same exact-equality bar the other block-map tests use. This file is named to
be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from sred_b200 import _lib, clutils, synth, utils

pytestmark = pytest.mark.gpu

METRICS = clutils.BLOCK_METRICS + [clutils.COSINE]


def _noalloc(metric, d_img, w, h, frames, ref, normalize, d_out, torch):
    L = _lib.load()
    st = L.sred_block_map_2d_device_noalloc(
        metric.encode(), C.c_void_p(d_img.data_ptr()), w, h, frames,
        np.ascontiguousarray(ref.pixels, np.float32), int(ref.size), ref.width, ref.height, float(ref.mean),
        float(ref.std), int(normalize), C.c_void_p(d_out.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st


@pytest.mark.parametrize("normalize", [True, False])
@pytest.mark.parametrize("metric", METRICS)
def test_noalloc_matches_regular_entry_point(metric, normalize):
    torch = pytest.importorskip("torch")
    ctx = _lib.Context(0, "fp32")
    w, h, frames = 61, 47, 3
    inputs = []
    for seed in (31, 32):  # two calls in a row, different data
        stack = np.stack([synth.normalize_input(synth.spot_image(w, h, 4, seed=seed + 10 * f))
                          for f in range(frames)])
        inputs.append(stack)
    ref = utils.get_reference_block_2d(inputs[0][0][10:19, 20:27])  # 9x7 block
    for stack in inputs:
        d_img = torch.from_numpy(stack).cuda()
        d_out = torch.full_like(d_img, float("nan"))
        assert _noalloc(metric, d_img, w, h, frames, ref, normalize, d_out, torch) == _lib.OK
        got = d_out.cpu().numpy()
        d_exp = torch.empty_like(d_img)
        clutils.block_map_device(metric, d_img.data_ptr(), w, h, frames, ref, 0.0, normalize, d_exp.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream, ctx=ctx)
        torch.cuda.synchronize()
        assert np.array_equal(got, d_exp.cpu().numpy()), metric
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    ref = utils.get_reference_block_2d(np.arange(9, dtype=np.float32).reshape(3, 3))
    d = torch.zeros(4097 * 9, device="cuda")
    assert _noalloc("SSIM", d, 3, 3, 4097, ref, True, d, torch) == _lib.ERR_ARG  # more than 4096 frames
    d = torch.zeros(1025 * 1025, device="cuda")
    assert _noalloc("NRMSE (inverted)", d, 1025, 1025, 1, ref, True, d, torch) == _lib.ERR_ARG
    assert _noalloc("nope", d, 1025, 1025, 1, ref, True, d, torch) == _lib.ERR_UNKNOWN_METRIC
    # a block whose image tile with halo needs more than 48 KB of shared memory
    L = _lib.load()
    k = L.sred_block_size(3, 401)
    tall = utils.ReferenceBlock2D(np.zeros(k, np.float32), 3, 401, 1, 200, k, 0.0, 1.0)
    assert _noalloc("Pearson's R", d, 1025, 1025, 1, tall, True, d, torch) == _lib.ERR_ARG
