"""Variance stabilisation on the GPU: the transform (bit-exact against the
restatement of java/VarianceStabilisingTransform2D_.java:136-151), the fit's
objective (java/GATMinimizer2D.java, relative 1e-12 against the restatement)
and the fit itself (a minimiser of that objective: at least as good as the
generating parameters, far better than the reference's starting point)."""
import numpy as np
import pytest

import oracle
from sred_b200 import _lib, utils
from tests.test_oracle import _poisson_gaussian

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return _lib.Context(0, "fp32")


def test_gat_transform_bitexact(ctx):
    img = _poisson_gaussian(130, 97, 2.0, 5.0, 100.0, 3)
    img[0, :4] = [-1e6, -50.0, 0.0, 1.0]
    for g, s, o in [(2.0, 5.0, 100.0), (1.0, 10.0, 100.0), (0.5, 30.0, -20.0)]:
        np.testing.assert_array_equal(utils.get_gat_2d(img, g, s, o, ctx=ctx), oracle.gat(img, g, s, o))


def test_gat_objective(ctx):
    img = _poisson_gaussian(257, 181, 2.0, 5.0, 100.0, 4)
    for g, s, o in [(2.0, 5.0, 100.0), (1.0, 10.0, 100.0), (3.0, 1.0, 50.0)]:
        a = utils.gat_objective_2d(img, g, s, o, ctx=ctx)
        b = oracle.gat_objective(img, g, s, o)
        assert abs(a - b) <= 1e-12 * abs(b), (a, b)
    tiny = np.zeros((5, 10), np.float32)  # blocks of height 5 // 6 = 0 (the reference divides by zero)
    with pytest.raises(_lib.SredError) as e:
        utils.gat_objective_2d(tiny, 1.0, 1.0, 0.0, ctx=ctx)
    assert e.value.status == _lib.ERR_ARG


def test_gat_fit_minimises_the_objective(ctx):
    img = _poisson_gaussian(384, 288, 2.0, 5.0, 100.0, 5)
    gain, sigma, offset, err = utils.fit_gat_2d(img, 5000, ctx=ctx)
    truth = oracle.gat_objective(img, 2.0, 5.0, 100.0)
    start = oracle.gat_objective(img, 1.0, 10.0, 100.0)
    assert abs(oracle.gat_objective(img, gain, sigma, offset) - err) <= 1e-12 * max(err, 1e-300)
    assert err <= truth * (1 + 1e-9) and err < start / 10, (gain, sigma, offset, err, truth, start)
    inp = utils.get_input_image_2d(img, True, True, "Simplex", 2000, ctx=ctx)
    assert inp.image_array.min() >= 0.0 and inp.image_array.max() <= 1.0


def test_gat_3d(ctx):
    """java/GATMinimizer3D.java: the objective (NaN outside its domain, grid
    halving for thin volumes), the transform over every voxel, the fit from
    the 3D command's start (gain 0: an objective of NaN)."""
    from tests.test_oracle import _poisson_gaussian3d
    vol = _poisson_gaussian3d(72, 60, 48, 2.0, 5.0, 100.0, 7)
    # Each block's variance is sum(v^2)/n - mean^2 with mean^2 ~ 1e3 and the
    # variance ~ 1: the GPU's tree-ordered FP64 sums and the reference's
    # sequential ones differ by ~1e-13 absolute in the variance, ~1e-11
    # relative in an objective of ~2e-3 near the optimum.
    for g, s, o in [(2.0, 5.0, 100.0), (1.0, 10.0, 100.0), (0.0, 100.0, 0.0), (1.0, -1.0, 3.0)]:
        a = utils.gat_objective_3d(vol, g, s, o, ctx=ctx)
        b = oracle.gat_objective3d(vol, g, s, o)
        assert (np.isnan(a) and np.isnan(b)) or abs(a - b) <= 1e-10 * abs(b), (g, s, o, a, b)
    # depth 5: blocks one slice deep; depth 1: an axis that can never hold two
    # blocks (the reference's grid loop never ends; here it stops)
    for thin in (vol[:5, :40, :9].copy(), vol[:1, :40, :9].copy()):
        for g, s, o in [(2.0, 5.0, 100.0), (0.7, 3.0, 20.0)]:
            a = utils.gat_objective_3d(thin, g, s, o, ctx=ctx)
            assert abs(a - oracle.gat_objective3d(thin, g, s, o)) <= 1e-10 * abs(a)
    np.testing.assert_array_equal(utils.get_gat_3d(vol, 2.0, 5.0, 100.0, ctx=ctx),
                                  oracle.gat(vol.reshape(-1, vol.shape[2]), 2.0, 5.0, 100.0).reshape(vol.shape))
    gain, sigma, offset, err = utils.fit_gat_3d(vol, 5000, ctx=ctx)
    assert abs(oracle.gat_objective3d(vol, gain, sigma, offset) - err) <= 1e-10 * max(err, 1e-300)
    assert err <= oracle.gat_objective3d(vol, 2.0, 5.0, 100.0) * (1 + 1e-9), (gain, sigma, offset, err)
    inp = utils.get_input_image_3d(vol, True, True, ctx=ctx)
    assert inp.depth == 48 and 0.0 <= inp.image_array.min() and inp.image_array.max() <= 1.0
