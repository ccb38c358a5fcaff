"""The pipelined host-stack block map (sred_block_map_2d_stack).

Chunks of frames move through two device slots with their uploads, maps and
downloads overlapping on three streams. Bar: every frame bit-equal to the
per-frame block map (sred_calculate_block_repetition_map_2d) for every
metric, relevance constant and chunk size (ragged last chunks included),
with pageable and page-locked host buffers; the time-lapse command of
java/BlockRepetition2D_.java:95-130 goes through it.
"""
import numpy as np
import pytest

from sred_b200 import _lib, clutils, plugins, synth, utils

pytestmark = pytest.mark.gpu

METRICS = clutils.BLOCK_METRICS + clutils.EXTRA_BLOCK_METRICS


@pytest.fixture(scope="module")
def ctx():
    return _lib.Context(0, "fp32")


def _stack(frames, h=40, w=52):
    return np.stack([synth.normalize_input(synth.spot_image(w, h, 5, seed=s)) for s in range(frames)])


@pytest.mark.parametrize("metric", METRICS)
def test_stack_equals_frame_by_frame(ctx, metric):
    st = _stack(5)
    _, h, w = st.shape
    rb = utils.get_reference_block_2d(st[0, 10:15, 20:25])
    for relc in (0.0, 1.0):
        one = [clutils.calculate_block_repetition_map_2d(metric, utils.InputImage2D(st[f].ravel(), w, h), rb, relc,
                                                         True, ctx=ctx) for f in range(5)]
        for chunk in (0, 1, 2, 5, 7):
            got = clutils.block_map_stack(metric, st, rb, relc, True, chunk_frames=chunk, ctx=ctx)
            assert got.shape == st.shape
            for f in range(5):
                np.testing.assert_array_equal(got[f].ravel(), one[f], err_msg=f"{metric} c={relc} chunk={chunk} f={f}")


def test_stack_page_locked_buffers_and_command(ctx):
    import torch
    st = _stack(9, 64, 80)
    rb = utils.get_reference_block_2d(st[0, 20:29, 30:39])
    h_in = torch.from_numpy(st).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    got = clutils.block_map_stack("Pearson's R", h_in.numpy(), rb, 0.0, True, chunk_frames=2, out=h_out.numpy(),
                                  ctx=ctx)
    assert np.shares_memory(got, h_out.numpy())
    exp = clutils.block_map_stack("Pearson's R", st, rb, 0.0, True, ctx=ctx)  # pageable, one chunk
    np.testing.assert_array_equal(h_out.numpy(), exp)
    # the time-lapse command: raw frames, each normalised on its own
    raw = (st * 1000.0 + 100.0).astype(np.float32)
    block = raw[0, 20:29, 30:39]
    cmd = plugins.block_repetition_2d(block, raw, 0.0, "SSIM", ctx=ctx)
    for f in range(raw.shape[0]):
        np.testing.assert_array_equal(cmd[f], plugins.block_repetition_2d(block, raw[f], 0.0, "SSIM", ctx=ctx))


def test_stack_errors(ctx):
    st = _stack(2)
    rb = utils.get_reference_block_2d(st[0, 10:15, 20:25])
    assert clutils.block_map_stack("nope", st, rb, 0.0, True, ctx=ctx) is None
    with pytest.raises(_lib.SredError):
        clutils.block_map_stack("Pearson's R", st, rb, 0.0, True, chunk_frames=-1, ctx=ctx)
    with pytest.raises(_lib.SredError):  # no frames
        clutils.block_map_stack("Pearson's R", st[:0], rb, 0.0, True, ctx=ctx)
    # a block wider than the frames leaves no interior: the same maps as frame by frame
    small = np.ascontiguousarray(st[:, :4, :4])
    got = clutils.block_map_stack("Pearson's R", small, rb, 0.0, True, ctx=ctx)
    for f in range(2):
        one = clutils.calculate_block_repetition_map_2d("Pearson's R", utils.InputImage2D(small[f].ravel(), 4, 4), rb,
                                                        0.0, True, ctx=ctx)
        np.testing.assert_array_equal(got[f].ravel(), one)


def test_frame_sharded_stack_on_one_gpu(ctx):
    """Each of three ranks' frame shards, mapped in turn on one GPU
    (block_map_stack_sharded without the gather), put together equals the
    whole stack mapped at once."""
    st = _stack(7)
    rb = utils.get_reference_block_2d(st[0, 10:15, 20:25])
    whole = clutils.block_map_stack("SSIM", st, rb, 1.0, True, ctx=ctx)
    parts = [clutils.block_map_stack_sharded("SSIM", st, rb, 1.0, True, r, 3, gather=False, ctx=ctx)
             for r in range(3)]
    assert [(f0, f1) for f0, f1, _ in parts] == [(0, 2), (2, 4), (4, 7)]
    np.testing.assert_array_equal(np.concatenate([m for _, _, m in parts]), whole)
