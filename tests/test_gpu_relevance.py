"""Parity of the relevance-mask tools through the C ABI.

References: the tools' kernels (cl/kernelGetRelevanceMask2D.cl,
cl/kernelGetLocalMeans.cl) compiled for the CPU, frozen in
tests/golden/relevance_refshim.npz, and the oracle's restatement of the Java
steps around them (tile noise variance in FP32 or FP64, thresholds, masks, the
OptimiseRelevanceMask_ loop run literally mask by mask).

Bar: bit-exact (masks, thresholds, noise variances, constants, range).
"""
import numpy as np
import pytest

import oracle
from sred_b200 import _lib, clutils, plugins, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return _lib.Context(0, "fp32")


def _cases(fx):
    for name in sorted({k.split("/")[0] for k in fx}):
        yield name, fx[f"{name}/image"], int(name.rsplit("x", 1)[1])


def test_relevance_mask_tool_bit_exact(ctx, relevance_fx):
    big = synth.normalize_input(synth.spot_image(400, 300, 24, seed=8))  # above CIF: 16x16 noise tiles
    cases = list(_cases(relevance_fx)) + [("big400x300_5x5", big, 5)]
    for name, img, b in cases:
        std = relevance_fx[f"{name}/std"] if f"{name}/std" in relevance_fx else oracle.local_var2d(img, b, b, 1)
        nv = oracle.tool_noise_var(img, 1)
        for c in (0.0, 0.5, 2.0, 10.0):
            rm = clutils.relevance_mask_tool_2d(img, b, b, c, ctx=ctx)
            assert rm.noise_mean_variance == nv, name
            assert rm.relevance_threshold == (np.float32(c) if nv == 0 else nv * np.float32(c)), name
            assert np.array_equal(rm.relevance_mask, oracle.tool_mask(std, b, b, nv, c)), (name, c)


def test_relevance_mask_sweep_bit_exact(ctx, relevance_fx):
    for name, img, b in _cases(relevance_fx):
        var = relevance_fx[f"{name}/var"]
        nv = oracle.tool_noise_var(img, 0)
        masks, consts, nv_gpu = clutils.relevance_mask_sweep_2d(img, b, b, 0.0, 0.1, 11, ctx=ctx)
        assert nv_gpu == nv
        c = np.float32(0.0)
        for i in range(11):
            assert consts[i] == c
            assert np.array_equal(masks[i], oracle.tool_mask(var, b, b, nv, c)), (name, i)
            c = np.float32(c + np.float32(0.1))


def test_relevance_constant_range_bit_exact(ctx, relevance_fx):
    for name, img, b in _cases(relevance_fx):
        var = relevance_fx[f"{name}/var"]
        nv = oracle.tool_noise_var(img, 0)
        for step in (1.0, 0.05, 0.013):
            ones, zeros, nv_gpu = clutils.relevance_constant_range_2d(img, b, b, step, ctx=ctx)
            assert nv_gpu == nv
            assert (ones, zeros) == oracle.tool_range(var, b, b, nv, step), (name, step)


def test_relevance_tools_zero_noise_and_errors(ctx):
    # flat tiles: noise variance 0, threshold = the constant itself
    img = np.zeros((48, 64), np.float32)
    img[8:40, 16:48] = synth.normalize_input(synth.spot_image(32, 32, 3, seed=2))
    var = oracle.local_var2d(img, 3, 3, 0)
    assert oracle.tool_noise_var(img, 0) == 0.0
    rm = clutils.relevance_mask_tool_2d(img, 3, 3, 1e-4, ctx=ctx)
    assert rm.noise_mean_variance == 0.0 and rm.relevance_threshold == np.float32(1e-4)
    assert np.array_equal(rm.relevance_mask, oracle.tool_mask(oracle.local_var2d(img, 3, 3, 1), 3, 3, 0.0, 1e-4))
    ones, zeros, _ = clutils.relevance_constant_range_2d(img, 3, 3, 1e-5, ctx=ctx)
    assert (ones, zeros) == oracle.tool_range(var, 3, 3, 0.0, 1e-5, max_iter=10 ** 6)
    with pytest.raises(_lib.SredError):  # the constant never grows: the reference loops forever
        clutils.relevance_constant_range_2d(img, 3, 3, 0.0, ctx=ctx)
    with pytest.raises(_lib.SredError):
        clutils.relevance_mask_sweep_2d(img, 3, 3, 0.0, 0.1, 0, ctx=ctx)
    with pytest.raises(_lib.SredError):  # smaller than one noise tile
        clutils.relevance_mask_tool_2d(np.ones((6, 6), np.float32), 3, 3, 1.0, ctx=ctx)


def test_relevance_commands_end_to_end(ctx):
    """The commands on a raw Poisson-Gaussian image: GAT fitted from gain 0,
    transform, FP64 normalisation, then the tool."""
    rng = np.random.default_rng(4)
    lam = synth.spot_image(96, 80, 6, seed=5, read_noise=0.0).clip(0, None) / 4.0
    raw = (2.0 * rng.poisson(lam) + 100.0 + rng.normal(0, 5.0, lam.shape)).astype(np.float32)
    inp = plugins.relevance_tools_input(raw, ctx=ctx)
    assert np.isfinite(inp).all() and inp.min() == 0.0 and inp.max() <= 1.0
    rm = plugins.relevance_mask_2d(raw, 3, 3, 1.0, ctx=ctx)
    exp = oracle.tool_mask(oracle.local_var2d(inp, 3, 3, 1), 3, 3, oracle.tool_noise_var(inp, 1), 1.0)
    assert np.array_equal(rm.relevance_mask, exp)
    masks, consts, inp2 = plugins.relevance_mask_stack_2d(raw, ctx=ctx)
    assert masks.shape == (11, 80, 96) and np.array_equal(inp2, inp)
    ones, zeros = plugins.optimise_relevance_mask(raw, step=0.5, ctx=ctx)
    assert 0.0 <= ones < zeros
