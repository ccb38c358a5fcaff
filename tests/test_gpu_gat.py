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


def _pg_spots(shape, seed):
    from sred_b200 import synth
    rng = np.random.default_rng(seed)
    if len(shape) == 2:
        lam = synth.spot_image(shape[1], shape[0], 8, seed=seed, read_noise=0.0).clip(0, None) / 4
    else:
        # dense, bright spots: the octree's Fisher test (width*height - 1
        # degrees of freedom for a whole block of voxels) splits the root
        lam = synth.spot_volume(shape[2], shape[1], shape[0], 6, 4, seed=seed, read_noise=0.0).clip(0, None)
    return (2.0 * rng.poisson(lam) + 100.0 + rng.normal(0, 5.0, lam.shape)).astype(np.float32)


@pytest.mark.parametrize("shape", [(96, 128), (200, 160), (36, 40, 48)])
def test_gat_tree_matches_restatement(ctx, shape):
    """QuadTree_ / OcTree_ against the oracle's literal FP32 restatement: the
    same leaves; g0, eDC and the transformed image within the difference of
    FP32 (reference) and FP64 (here) sums."""
    img = _pg_spots(shape, 3 + len(shape))
    octree = len(shape) == 3
    r = oracle.gat_tree(img, octree=octree)
    if octree:
        out, g0, edc, nl = utils.gat_octree_3d(img, ctx=ctx)
    else:
        out, g0, edc, nl = utils.gat_quadtree_2d(img, ctx=ctx)
    assert nl == len(r["boxes"])
    assert abs(g0 - r["g0"]) <= 2e-3 * abs(r["g0"]) and abs(edc - r["edc"]) <= 2e-3 * abs(r["edc"]), (g0, edc, r)
    ref = r["image"]
    assert float(np.max(np.abs(out - ref) / np.maximum(np.abs(ref), 1.0))) <= 2e-3


def test_gat_tree_in_input_images(ctx):
    img = _pg_spots((96, 128), 9)
    inp = utils.get_input_image_2d(img, True, True, "Quad/Octree", ctx=ctx)
    assert inp.image_array.min() == 0.0 and inp.image_array.max() <= 1.0
    vol = _pg_spots((24, 40, 48), 10)
    inp3 = utils.get_input_image_3d(vol, True, True, "Quad/Octree", ctx=ctx)
    assert inp3.depth == 24 and np.isfinite(inp3.image_array).all()
    with pytest.raises(_lib.SredError):
        utils.gat_quadtree_2d(img, min_size=0, ctx=ctx)
    # every leaf with the same mean: no regression line (the reference goes on with NaN)
    flat = np.full((16, 24, 24), 100.0, np.float32)
    with pytest.raises(ValueError):
        oracle.gat_tree(flat, octree=True)
    with pytest.raises(_lib.SredError):
        utils.gat_octree_3d(flat, ctx=ctx)


def test_variance_stabilising_commands(ctx):
    """VarianceStabilisingTransform2D_ / 3D_: the Simplex fit from the dialog's
    guesses (gain 1, offset 10, noise std 100) or from a ROI estimate, then
    getGAT with the fitted parameters; the 3D command refuses single slices."""
    from sred_b200 import plugins
    from tests.test_oracle import _poisson_gaussian3d
    img = _poisson_gaussian(200, 150, 2.0, 5.0, 100.0, 9)
    out, g, s, o = plugins.variance_stabilising_transform_2d(img, max_iterations=3000, ctx=ctx)
    assert (g, s, o) == utils.fit_gat_2d(img, 3000, 1.0, 100.0, 10.0, ctx=ctx)[:3]
    np.testing.assert_array_equal(out, oracle.gat(img, g, s, o))
    assert oracle.gat_objective(img, g, s, o) < oracle.gat_objective(img, 1.0, 100.0, 10.0) / 10
    roi = (10, 20, 30, 25)
    off, sd = plugins.roi_offset_and_sigma(img, roi)
    out2, g2, s2, o2 = plugins.variance_stabilising_transform_2d(img, roi=roi, max_iterations=3000, ctx=ctx)
    assert (g2, s2, o2) == utils.fit_gat_2d(img, 3000, 1.0, sd, off, ctx=ctx)[:3]
    np.testing.assert_array_equal(out2, oracle.gat(img, g2, s2, o2))
    vol = _poisson_gaussian3d(40, 36, 12, 2.0, 5.0, 100.0, 10)
    v3, g3, s3, o3 = plugins.variance_stabilising_transform_3d(vol, max_iterations=2000, ctx=ctx)
    assert (g3, s3, o3) == utils.fit_gat_3d(vol, 2000, 1.0, 100.0, 10.0, ctx=ctx)[:3]
    np.testing.assert_array_equal(v3, utils.get_gat_3d(vol, g3, s3, o3, ctx=ctx))
    with pytest.raises(ValueError):
        plugins.variance_stabilising_transform_3d(vol[:1], ctx=ctx)
