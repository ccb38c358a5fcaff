"""Parity of the shape metrics (Hu moments, phase correlation) through the C ABI.

References: the reference's shape kernels compiled for the CPU
(cl/kernelGetPatchHu2D.cl, cl/kernelGetHuMap.cl, and
cl/kernelGetPhaseCorrelationMap.cl with its three defects repaired), frozen
in tests/golden/shape_refshim.npz, and the oracle's restatements of them.

Bars:
  * Hu patch map (FP64 in both): within 2 float ulps of the reference kernel
    (pow(x, 2.0) there, x * x here);
  * Hu map (FP32 terms): relative 2e-6 against the FP64-accumulated judge of
    the reference's own FP32 terms, 2e-5 against the reference's FP32 sums;
  * phase correlation (FP64): every peak decision equal to the judge's, so the
    sums agree to FP32 rounding of the result (relative 2e-7), and within the
    reference's own FP32 accumulation error (2e-5) of its sums;
  * block-map forms: raw maps against the oracle as above (phase: equal),
    post-processed maps within 1e-6.
"""
import numpy as np
import pytest

import oracle
from sred_b200 import _lib, clutils, utils

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return _lib.Context(0, "fp32")


def _cases(fx):
    for n in sorted({k.split("/")[0] for k in fx}):
        bw, bh = (int(v) for v in n.rsplit("_", 1)[1].split("x"))
        yield n, bw, bh


def _inp(img):
    h, w = img.shape
    return utils.InputImage2D(np.ascontiguousarray(img, np.float32), w, h)


def _stats(img, bw, bh):
    m, s = oracle.local_stats(img, bw, bh)
    return clutils.CLLocalStatistics(m.ravel(), s.ravel())


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))


def test_patch_hu_matches_reference_kernel(ctx, shape_fx):
    for name, bw, bh in _cases(shape_fx):
        img = shape_fx[f"{name}/image"]
        got = clutils.get_patch_hu_map_2d(_inp(img), shape_fx[f"{name}/patch_hu/patch"], bw, bh, ctx=ctx)
        assert _rel(got, shape_fx[f"{name}/patch_hu/map"]) <= 2.5e-7, name


def test_hu_map_matches_reference_kernel(ctx, shape_fx):
    for name, bw, bh in _cases(shape_fx):
        img = shape_fx[f"{name}/image"]
        got = clutils.get_hu_map_2d(_inp(img), _stats(img, bw, bh), bw, bh, ctx=ctx)
        assert _rel(got, oracle.hu_map(img, bw, bh, precision="f64")) <= 2e-6, name
        assert _rel(got, shape_fx[f"{name}/hu_map"]) <= 2e-5, name


def test_phase_map_matches_reference_kernel(ctx, shape_fx):
    n = 0
    for name, bw, bh in _cases(shape_fx):
        if f"{name}/phase_map" not in shape_fx:
            continue
        img = shape_fx[f"{name}/image"]
        got = clutils.get_phase_correlation_map_2d(_inp(img), _stats(img, bw, bh), bw, bh, ctx=ctx)
        judge = oracle.phase_map(img, bw, bh, precision="f64")
        assert _rel(got, judge.astype(np.float32)) <= 2e-7, name
        assert _rel(got, shape_fx[f"{name}/phase_map"]) <= 2e-5, name
        n += 1
    assert n >= 3


def _block(fx, name, bw, bh):
    px = fx[f"{name}/block/pixels"]
    m, s = fx[f"{name}/block/mean_std"]
    return utils.ReferenceBlock2D(px, bw, bh, bw // 2, bh // 2, px.size, float(m), float(s))


@pytest.mark.parametrize("metric", [clutils.HU, clutils.PHASE])
def test_block_shape_metrics(ctx, shape_fx, metric):
    for name, bw, bh in _cases(shape_fx):
        img = shape_fx[f"{name}/image"]
        H, W = img.shape
        rb = _block(shape_fx, name, bw, bh)
        raw = clutils.calculate_block_repetition_map_2d(metric, _inp(img), rb, 0.0, False, ctx=ctx)
        if metric == clutils.HU:
            patch = oracle.hu_prepare_patch(rb.pixels, bw, bh)
            exp = oracle.patch_hu_map(patch, img, bw, bh)
            assert _rel(raw, exp) <= 2.5e-7, name
        else:
            exp = oracle.block_phase_raw(img, rb.pixels, bw, bh, rb.std).astype(np.float32)
            np.testing.assert_array_equal(raw, exp.ravel(), err_msg=name)
        # post-processing as Pearson's: relevance mask, min-max normalisation
        _, stds = oracle.local_stats(img, bw, bh)
        for c in (0.0, 1.0):
            got = clutils.calculate_block_repetition_map_2d(metric, _inp(img), rb, c, True, ctx=ctx)
            a = np.ascontiguousarray(exp, np.float32).ravel().copy()
            rc = oracle.lib().orc_block_postprocess_f32(0, a, np.ascontiguousarray(img, np.float32), W, H,
                                                        bw // 2, bh // 2, stds, np.float32(c), 1)
            assert rc == 0
            np.testing.assert_allclose(got, a, atol=1e-6, rtol=0, err_msg=f"{name} c={c}")


def test_block_hu_distance(ctx, shape_fx):
    """Block-map Hu distance (the L2 distance of the seven Hu invariants to the
    reference block's; this library's metric, the reference outputs Hu1 only):
    the raw map within 1e-6 of the FP64 oracle on every shape fixture (relative
    to the map's largest distance), about 0 at the reference block's own
    position, frame stacks equal to single frames, and the post-processing of
    the other block metrics (relevance mask, min-max normalisation)."""
    from sred_b200 import synth
    for name, bw, bh in _cases(shape_fx):
        img = shape_fx[f"{name}/image"]
        H, W = img.shape
        rb = _block(shape_fx, name, bw, bh)
        raw = clutils.calculate_block_repetition_map_2d(clutils.HU7, _inp(img), rb, 0.0, False, ctx=ctx)
        exp, _ = oracle.block_hu7_raw(img, rb.pixels[:rb.size], bw, bh)
        scale = float(np.max(exp))
        assert scale > 0 and float(np.max(np.abs(raw - exp.ravel()))) <= 1e-6 * scale, name
        _, stds = oracle.local_stats(img, bw, bh)
        for c in (0.0, 1.0):
            got = clutils.calculate_block_repetition_map_2d(clutils.HU7, _inp(img), rb, c, True, ctx=ctx)
            a = np.ascontiguousarray(exp, np.float32).ravel().copy()
            rc = oracle.lib().orc_block_postprocess_f32(0, a, np.ascontiguousarray(img, np.float32), W, H,
                                                        bw // 2, bh // 2, stds, np.float32(c), 1)
            assert rc == 0
            np.testing.assert_allclose(got, a, atol=2e-6, rtol=0, err_msg=f"{name} c={c}")
    img = synth.normalize_input(synth.spot_image(45, 37, 6, seed=77))
    rb = utils.get_reference_block_2d(img[15:24, 18:27])  # 9 x 9 centred at (19, 22)
    raw = clutils.calculate_block_repetition_map_2d(clutils.HU7, _inp(img), rb, 0.0, False, ctx=ctx).reshape(37, 45)
    assert raw[19, 22] <= 1e-6 * float(raw.max())
    torch = pytest.importorskip("torch")
    stack = np.stack([img, img[::-1].copy()])
    d_in = torch.from_numpy(stack).cuda()
    d_out = torch.empty_like(d_in)
    clutils.block_map_device(clutils.HU7, d_in.data_ptr(), 45, 37, 2, rb, 0.0, False, d_out.data_ptr(), ctx=ctx)
    torch.cuda.synchronize()
    for f in range(2):
        single = clutils.calculate_block_repetition_map_2d(clutils.HU7, _inp(stack[f]), rb, 0.0, False, ctx=ctx)
        assert np.array_equal(d_out[f].cpu().numpy().ravel(), single), f


@pytest.mark.parametrize("bw,bh", [(7, 7), (11, 9), (13, 13), (15, 15), (15, 7), (3, 15), (5, 11)])
def test_block_phase_every_block_size(ctx, bw, bh):
    """The block-map phase kernel is instantiated per max(bw, bh) (3 ... 15),
    with 4, 8 or 16 lanes per pixel; every size equals the FP64 oracle. The
    45 x 37 plane is not a multiple of the 128 pixels of a CTA."""
    from sred_b200 import synth
    img = synth.normalize_input(synth.spot_image(45, 37, 6, seed=bw * 31 + bh))
    cy, cx = 18, 22
    rb = utils.get_reference_block_2d(img[cy - bh // 2:cy + bh // 2 + 1, cx - bw // 2:cx + bw // 2 + 1])
    raw = clutils.calculate_block_repetition_map_2d(clutils.PHASE, _inp(img), rb, 0.0, False, ctx=ctx)
    exp = oracle.block_phase_raw(img, rb.pixels, bw, bh, rb.std).astype(np.float32)
    assert np.count_nonzero(exp) > 0
    np.testing.assert_array_equal(raw, exp.ravel(), err_msg=f"{bw}x{bh}")


@pytest.mark.parametrize("metric", [clutils.HU, clutils.PHASE, clutils.HU7])
def test_block_shape_frames_and_noalloc(ctx, shape_fx, metric):
    """A stack of frames on the device equals the frames one by one; the
    allocation-free entry point gives the same maps."""
    import torch
    name, bw, bh = "spots32x28_3x3", 3, 3
    img = shape_fx[f"{name}/image"]
    img2 = np.ascontiguousarray(img[::-1, :])
    rb = _block(shape_fx, name, bw, bh)
    H, W = img.shape
    d_in = torch.from_numpy(np.stack([img, img2])).cuda()
    d_out = torch.empty_like(d_in)
    clutils.block_map_device(metric, d_in.data_ptr(), W, H, 2, rb, 0.0, True, d_out.data_ptr(), ctx=ctx)
    torch.cuda.synchronize()
    for f, im in enumerate((img, img2)):
        one = clutils.calculate_block_repetition_map_2d(metric, _inp(im), rb, 0.0, True, ctx=ctx)
        np.testing.assert_array_equal(d_out[f].cpu().numpy().ravel(), one)
    d_na = torch.empty_like(d_in)
    L = _lib.load()
    st = L.sred_block_map_2d_device_noalloc(metric.encode(), d_in.data_ptr(), W, H, 2,
                                            np.ascontiguousarray(rb.pixels, np.float32), int(rb.size), bw, bh,
                                            float(rb.mean), float(rb.std), 1, d_na.data_ptr(), None)
    assert st == _lib.OK
    torch.cuda.synchronize()
    assert torch.equal(d_na, d_out)


def test_shape_argument_errors(ctx, shape_fx):
    img = shape_fx["spots32x28_3x3/image"]
    with pytest.raises(_lib.SredError) as e:
        clutils.get_phase_correlation_map_2d(_inp(img), _stats(img, 3, 3), 17, 3, ctx=ctx)
    assert e.value.status == _lib.ERR_ARG
    tiny = np.zeros((4, 4), np.float32)
    with pytest.raises(_lib.SredError) as e:
        clutils.get_hu_map_2d(_inp(tiny), _stats(tiny, 5, 5), 5, 5, ctx=ctx)
    assert e.value.status == _lib.ERR_ARG


def test_hu_map_constant_image(ctx):
    """A constant image: every block's feature is 0 / (0 + eps) = 0 and every
    term vanishes, so the map is exactly 0."""
    img = np.full((20, 24), 0.25, np.float32)
    got = clutils.get_hu_map_2d(_inp(img), _stats(img, 3, 3), 3, 3, ctx=ctx)
    assert not np.any(got)


def test_fixed_divisor_division_fp64_is_ieee(ctx):
    """The FP64 div_fixed (Markstein's correction of a * RN(1/b)) that the
    block-map Hu kernel divides each block by, against IEEE float64 division
    on 4M numerators per divisor: uniform in [0, b] (the kernel's range),
    uniform in [0, 1], tiny (down to 1e-200), powers of two and exact
    multiples of the divisor; divisors like max - min + eps of normalised
    blocks and awkward significands."""
    rng = np.random.default_rng(22)
    base = np.concatenate([rng.random(1 << 21), 10.0 ** rng.uniform(-200, 0, 1 << 20),
                           2.0 ** rng.integers(-600, 1, 1 << 19).astype(np.float64), np.zeros(16)])
    for b in (1.0 + 1e-9, 0.37, 3.0e-3, 1.0e-6 + 1e-9, 0.9999999999999999, 1.0000000000000002,
              1.9999999999999998, 1.4142135623730951):
        aa = np.concatenate([base, base[: 1 << 21] * b, b * np.arange(1, 1 << 19, dtype=np.float64)])
        out = np.empty_like(aa)
        ctx.check(ctx._L.sred_debug_divide_fixed64(ctx.h, aa, aa.size, float(b), out), "sred_debug_divide_fixed64")
        exp = aa / b
        bad = np.flatnonzero(out.view(np.uint64) != exp.view(np.uint64))
        assert bad.size == 0, (b, aa[bad[:5]], out[bad[:5]], exp[bad[:5]])
