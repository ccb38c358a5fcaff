"""Redundancy classification (java/ClassifyRedundancy_.java) through the C ABI.

Reference: the oracle's restatement of the clusterer (k-means++ and Lloyd as
commons-math3 3.6.1 KMeansPlusPlusClusterer runs them, java.util.Random, and
the library's fixed summation order). The reference seeds its generator from
the clock, so only the algorithm is pinned, not a particular clustering.

Bar: bit-exact (class map, classes used, WCSS).
"""
import numpy as np
import pytest

import oracle
from sred_b200 import _lib, plugins, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return _lib.Context(0, "fp32")


@pytest.mark.parametrize("shape,border,k,seed", [((70, 90), 1, 3, 0), ((128, 160), 4, 5, 11),
                                                 ((64, 64), 0, 1, 3), ((200, 120), 2, 8, 99)])
def test_classify_bit_exact(ctx, shape, border, k, seed):
    h, w = shape
    m = synth.normalize_input(synth.spot_image(w, h, 6, seed=seed + 1))
    out, kc, wcss = plugins.classify_redundancy(m, border, k, seed=seed, ctx=ctx)
    eo, ek, ew = oracle.classify_redundancy(m, border, k, seed=seed)
    assert kc == ek == k and wcss == ew
    assert np.array_equal(out, eo)


def test_classify_elbow_and_large_map(ctx):
    m = synth.normalize_input(synth.image_1024_spots(seed=2))[:700, :900].copy()
    out, kc, wcss = plugins.classify_redundancy(m, 1, 3, optimal_k=True, max_k=6, seed=7, ctx=ctx)
    eo, ek, ew = oracle.classify_redundancy(m, 1, 3, True, 6, seed=7)
    assert kc == ek and wcss == ew and np.array_equal(out, eo)


def test_classify_degenerate_maps(ctx):
    # a constant map: every centre equal, empty clusters refilled each round
    flat = np.full((20, 24), 0.5, np.float32)
    out, kc, _ = plugins.classify_redundancy(flat, 1, 3, seed=1, ctx=ctx)
    eo, ek, _ = oracle.classify_redundancy(flat, 1, 3, seed=1)
    assert kc == ek and np.array_equal(out, eo)
    # two values only, three classes
    two = np.zeros((30, 30), np.float32)
    two[:, 15:] = 1.0
    out, kc, _ = plugins.classify_redundancy(two, 0, 3, seed=4, ctx=ctx)
    assert np.array_equal(out, oracle.classify_redundancy(two, 0, 3, seed=4)[0])
    with pytest.raises(_lib.SredError):  # no pixel left inside the border
        plugins.classify_redundancy(flat, 12, 3, ctx=ctx)
    with pytest.raises(_lib.SredError):
        plugins.classify_redundancy(flat, 1, 0, ctx=ctx)
