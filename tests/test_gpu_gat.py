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
