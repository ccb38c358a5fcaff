"""Parity of the CUDA path (through the C ABI) with the oracle.

Bars:
  * integer-like and reference-FP32 quantities (local statistics, noise
    variance, relevance masks, block maps): bit-exact with the reference's
    kernels compiled for the CPU (frozen fixtures) and the JUnit vectors;
  * global maps: max abs error on the normalised map against the FP64 judge
    within GLOBAL_TOL[engine], and against the reference's FP32 kernels
    within REF_TOL (the reference's own FP32 accumulation error is part of
    that difference).
"""
import json
import os

import numpy as np
import pytest

import oracle
from sred_b200 import _lib, clutils, plugins, synth, utils

pytestmark = pytest.mark.gpu

# Max abs error of the normalised global map against the FP64 judge.
GLOBAL_TOL = {"fp32": 1e-5, "tc": 1e-5}
# Against the reference's FP32 kernels (their own rounding included).
REF_TOL = 2e-5
ENGINES = ["fp32", "tc"]

_report = []


def _note(**kw):
    _report.append(kw)


@pytest.fixture(scope="module", autouse=True)
def report():
    yield
    path = os.environ.get("SRED_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            for r in _report:
                f.write(json.dumps(r, default=float) + "\n")


@pytest.fixture(scope="module")
def ctx():
    return _lib.Context(0, "fp32")


def _img_cases(fx):
    out = []
    for name in sorted({k.split("/")[0] for k in fx}):
        bw, bh = (int(v) for v in name.rsplit("_", 1)[1].split("x"))
        cs = sorted({float(k.split("/")[1][1:]) for k in fx if k.startswith(name + "/c")})
        out.append((name, bw, bh, cs))
    return out


def _junit_block(g):
    from tests.test_oracle import _ref_block_as_junit
    px, m, s = _ref_block_as_junit(g["block"], g["block_width"], g["block_height"])
    return utils.ReferenceBlock2D(px, g["block_width"], g["block_height"], g["block_width"] // 2,
                                  g["block_height"] // 2, px.size, m, s)


# --------------------------------------------------------------------------
# Moments, noise variance, relevance mask: bit-exact
# --------------------------------------------------------------------------

def test_local_statistics_golden(ctx, junit):
    g = junit["local_statistics_2d"]
    inp = utils.InputImage2D(np.array(g["image"], np.float32), g["width"], g["height"])
    st = clutils.get_local_statistics_2d(inp, 3, 3, ctx)
    np.testing.assert_allclose(st.local_means, g["expected_means"], atol=g["tolerance"], rtol=0)
    np.testing.assert_allclose(st.local_stds, g["expected_stds"], atol=g["tolerance"], rtol=0)


def test_local_statistics_bitexact(ctx, refshim_fx):
    for name, bw, bh, _ in _img_cases(refshim_fx):
        img = refshim_fx[f"{name}/image"]
        H, W = img.shape
        st = clutils.get_local_statistics_2d(utils.InputImage2D(img.ravel(), W, H), bw, bh, ctx)
        m, s = oracle.local_stats(img, bw, bh)
        assert np.array_equal(st.local_means, m.ravel()) and np.array_equal(st.local_stds, s.ravel()), name


def test_relevance_mask_golden(ctx, junit):
    g = junit["relevance_mask"]
    W, H = g["width"], g["height"]
    stream = oracle.java_random_floats(g["java_random_seed"], 2 * W * H)
    img = np.zeros(W * H, np.float32)
    stds = np.zeros(W * H, np.float32)
    k = 0
    for i in range(W * H):
        if i % 50 == 0:
            img[i], stds[i] = 1.0, 0.0
        else:
            img[i] = np.float32(1.0) + stream[k] * np.float32(2.0)
            stds[i] = stream[k + 1]
            k += 2
    rm = utils.get_relevance_mask(img, W, H, 2, 2, stds, g["relevance_constant"], ctx)
    assert rm.relevance_threshold == np.float32(g["expected_threshold"])
    assert float(rm.noise_mean_variance) == g["expected_noise_var"]
    m, thr, nv = oracle.relevance_mask(img.reshape(H, W), 5, 5, stds.reshape(H, W), g["relevance_constant"])
    assert np.array_equal(rm.relevance_mask, m.ravel())


def test_relevance_mask_bitexact(ctx, refshim_fx):
    for name, bw, bh, cs in _img_cases(refshim_fx):
        img = refshim_fx[f"{name}/image"]
        H, W = img.shape
        _, s = oracle.local_stats(img, bw, bh)
        for c in cs + [0.5, 3.0]:
            rm = utils.get_relevance_mask(img.ravel(), W, H, bw // 2, bh // 2, s.ravel(), c, ctx)
            m, thr, nv = oracle.relevance_mask(img, bw, bh, s, c)
            assert rm.relevance_threshold == thr and rm.noise_mean_variance == nv
            assert np.array_equal(rm.relevance_mask, m.ravel()), (name, c)


# --------------------------------------------------------------------------
# Block (local) maps
# --------------------------------------------------------------------------

@pytest.mark.parametrize("idx", range(4))
def test_block_map_golden(ctx, junit, idx):
    g = junit["block_maps_2d"][idx]
    inp = utils.InputImage2D(np.array(g["image"], np.float32), g["width"], g["height"])
    out = clutils.calculate_block_repetition_map_2d(g["metric"], inp, _junit_block(g), g["relevance_constant"],
                                                    g["normalize"], ctx=ctx)
    assert np.all((out >= 0) & (out <= 1))
    np.testing.assert_allclose(out, g["expected"], atol=g["tolerance"], rtol=0)


def test_block_map_all_metrics_range(ctx, junit):
    """src/test/java/CLUtilsTest.java testCalculateBlockRepetitionMap2DAllMetrics."""
    g = junit["block_maps_2d"][0]
    inp = utils.InputImage2D(np.array(g["image"], np.float32), 10, 10)
    for metric in clutils.BLOCK_METRICS:
        out = clutils.calculate_block_repetition_map_2d(metric, inp, _junit_block(g), 0.0, True, ctx=ctx)
        assert out is not None and out.size == 100
        assert np.all((out >= 0) & (out <= 1)), metric
    assert clutils.calculate_block_repetition_map_2d("nope", inp, _junit_block(g), 0.0, True, ctx=ctx) is None


def test_block_maps_bitexact_vs_reference_kernels(ctx, refshim_fx):
    fx = refshim_fx
    n = 0
    for name, bw, bh, _ in _img_cases(fx):
        img = fx[f"{name}/image"]
        H, W = img.shape
        px = fx[f"{name}/block/pixels"]
        bm, bs = fx[f"{name}/block/mean_std"]
        ref = utils.ReferenceBlock2D(px, bw, bh, bw // 2, bh // 2, px.size, bm, bs)
        for metric in clutils.BLOCK_METRICS:
            for c in (0.0, 1.0):
                out = clutils.calculate_block_repetition_map_2d(metric, utils.InputImage2D(img.ravel(), W, H),
                                                                ref, c, True, ctx=ctx)
                exp = fx[f"{name}/block/c{c:g}/{metric}/map"].ravel()
                d = float(np.max(np.abs(out - exp)))
                _note(test="block_bitexact", case=name, metric=metric, c=c, max_abs=d)
                assert np.array_equal(out, exp), (name, metric, c, d)
                n += 1
    assert n >= 40


def test_block_cosine_vs_fp64(ctx):
    img = synth.normalize_input(synth.spot_image(96, 80, 6, seed=21))
    ref = utils.get_reference_block_2d(img[30:45, 40:55])
    out = clutils.calculate_block_repetition_map_2d("Cosine", utils.InputImage2D(img.ravel(), 96, 80), ref, 0.0,
                                                    False, ctx=ctx)
    _, s = oracle.local_stats(img, 15, 15)
    exp = oracle.block_raw_f64(oracle.COSINE, img, ref.pixels, 15, 15, ref.mean, ref.std, s)
    err = float(np.max(np.abs(out - exp.ravel())))
    _note(test="block_cosine", max_abs=err)
    assert err < 2e-6


def test_block_map_stack(ctx, refshim_fx):
    """Frames of a stack are processed independently (the time-lapse loop)."""
    torch = pytest.importorskip("torch")
    fx = refshim_fx
    name = "spots48x40_3x3"
    img = fx[f"{name}/image"]
    H, W = img.shape
    px = fx[f"{name}/block/pixels"]
    bm, bs = fx[f"{name}/block/mean_std"]
    ref = utils.ReferenceBlock2D(px, 3, 3, 1, 1, px.size, bm, bs)
    stack = np.stack([img, img[::-1].copy(), img[:, ::-1].copy()])
    d_in = torch.from_numpy(stack).cuda()
    for metric in clutils.BLOCK_METRICS:
        for c in (0.0, 1.0):
            d_out = torch.empty_like(d_in)
            clutils.block_map_device(metric, d_in.data_ptr(), W, H, 3, ref, c, True, d_out.data_ptr(), ctx=ctx)
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            for f in range(3):
                exp = oracle.block_map(metric, stack[f], px, 3, 3, bm, bs, c, True)["map"]
                assert np.array_equal(got[f], exp), (metric, c, f)


# --------------------------------------------------------------------------
# Global maps
# --------------------------------------------------------------------------

def _global_gpu(ctx, engine, metric, img, bw, bh, c, normalize=True, dropin=False):
    ctx.set_engine(engine)
    if not dropin:
        out, info = clutils.global_map_host(metric, img, bw, bh, c, normalize, ctx=ctx)
        return out, info
    H, W = img.shape
    inp = utils.InputImage2D(img.ravel(), W, H)
    st = clutils.get_local_statistics_2d(inp, bw, bh, ctx)
    rm = utils.get_relevance_mask(inp.image_array, W, H, bw // 2, bh // 2, st.local_stds, c, ctx)
    npx = oracle.n_pixels(rm.relevance_mask.reshape(H, W), bw // 2, bh // 2)
    info = {}
    out = clutils.calculate_global_repetition_map_2d(metric, inp, bw, bh, utils.block_size(bw, bh), st, rm, npx,
                                                     normalize, ctx, info)
    return out.reshape(H, W), info


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("metric", clutils.GLOBAL_METRICS)
def test_global_vs_reference_and_fp64(ctx, refshim_fx, engine, metric):
    fx = refshim_fx
    for name, bw, bh, cs in _img_cases(fx):
        img = fx[f"{name}/image"]
        for c in cs:
            out, info = _global_gpu(ctx, engine, metric, img, bw, bh, c)
            ref = fx[f"{name}/c{c:g}/{metric}/map"]
            j = oracle.global_map(metric, img, bw, bh, c, precision="f64")
            e_ref = float(np.max(np.abs(out - ref)))
            e64 = float(np.max(np.abs(out - j["map"])))
            e_ref64 = float(np.max(np.abs(ref - j["map"])))
            _note(test="global_small", engine=engine, metric=metric, case=name, c=c, err_vs_ref32=e_ref,
                  err_vs_f64=e64, ref32_vs_f64=e_ref64)
            if not np.all(np.isfinite(ref)):
                # Degenerate input (noise variance 0, weights exp(-d^2/1e-7)):
                # the reference's FP32 inversion overflows where its per-pair
                # sums underflow; which pixels do depends on FP32 denormal
                # rounding of each term. The drop-in overflows too.
                assert not np.all(np.isfinite(out)), (name, c)
                continue
            # At least as close to FP64 as the reference's own FP32 kernels
            # (ill-conditioned weights make both deviate alike).
            assert e64 <= max(GLOBAL_TOL[engine], 1.25 * e_ref64), (name, c, e64)
            assert e_ref <= REF_TOL + e_ref64, (name, c, e_ref)


@pytest.mark.parametrize("engine", ENGINES)
def test_global_dropin_signature(ctx, refshim_fx, engine):
    """calculateGlobalRepetitionMap2D with caller-provided stats and mask."""
    img = refshim_fx["spots40x44_5x5/image"]
    for metric in clutils.GLOBAL_METRICS:
        a, _ = _global_gpu(ctx, engine, metric, img, 5, 5, 1.0, dropin=True)
        b, _ = _global_gpu(ctx, engine, metric, img, 5, 5, 1.0, dropin=False)
        assert np.array_equal(a, b), metric


def test_plugin_command_matches_dropin(ctx, refshim_fx):
    raw = synth.spot_image(52, 36, 5, seed=13)
    ctx.set_engine("fp32")
    a = plugins.global_repetition_2d(raw, 5, 3, 2.0, "SSIM", ctx=ctx)
    b, _ = _global_gpu(ctx, "fp32", "SSIM", synth.normalize_input(raw), 5, 3, 2.0)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("engine", ENGINES)
def test_global_edge_cases(ctx, engine):
    ctx.set_engine(engine)
    img = synth.normalize_input(synth.spot_image(40, 40, 3, seed=3))
    # unknown metric: None, as the reference's dispatch returns null
    inp = utils.InputImage2D(img.ravel(), 40, 40)
    st = clutils.get_local_statistics_2d(inp, 3, 3, ctx)
    rm = utils.get_relevance_mask(img.ravel(), 40, 40, 1, 1, st.local_stds, 0.0, ctx)
    assert clutils.calculate_global_repetition_map_2d("Pearson", inp, 3, 3, 5, st, rm, 1.0, True, ctx) is None
    # even block: rejected
    with pytest.raises(_lib.SredError) as ei:
        clutils.global_map_host("SSIM", img, 4, 3, 0.0, ctx=ctx)
    assert ei.value.status == _lib.ERR_ARG
    # image smaller than one noise tile: the reference indexes past its tile list
    with pytest.raises(_lib.SredError):
        clutils.global_map_host("SSIM", img[:6, :6].copy(), 3, 3, 0.0, ctx=ctx)
    # NaN in a noise tile
    bad = img.copy()
    bad[2, 2] = np.nan
    with pytest.raises(_lib.SredError) as ei:
        clutils.global_map_host("NRMSE", bad, 3, 3, 0.0, ctx=ctx)
    assert ei.value.status == _lib.ERR_INVALID_INPUT
    # every block masked out
    for metric in clutils.GLOBAL_METRICS:
        out, info = clutils.global_map_host(metric, img, 3, 3, 1e9, ctx=ctx)
        exp = oracle.global_map(metric, img, 3, 3, 1e9)["map"]
        assert info["n_relevant"] == 0
        assert np.array_equal(out, exp), metric
    # ragged sizes, non-square blocks, 1-pixel-wide interior
    for (h, w, bw, bh) in [(33, 17, 3, 5), (17, 40, 7, 3), (11, 23, 9, 9)]:
        im = synth.normalize_input(synth.spot_image(w, h, 2, seed=h + w))
        for metric in clutils.GLOBAL_METRICS:
            out, _ = clutils.global_map_host(metric, im, bw, bh, 0.0, ctx=ctx)
            exp = oracle.global_map(metric, im, bw, bh, 0.0, precision="f64")["map"]
            e = float(np.max(np.abs(out - exp)))
            _note(test="global_ragged", engine=engine, metric=metric, shape=(h, w, bw, bh), err_vs_f64=e)
            assert e <= GLOBAL_TOL[engine], (h, w, bw, bh, metric, e)


# Relative error of the raw (unnormalised) map value per sampled row against
# the FP64 judge: num / (den nPixels + eps) (inverted for NRMSE), so that a
# wrong normalisation cannot cancel out.
RAW_TOL = {"fp32": 2e-6, "tc": 5e-6}


def _sampled_errors(ctx, out, info, img, metric, bw, bh, c, rows):
    """Errors of the GPU map on sampled reference pixels against the FP64 judge.

    Returns a dict: norm_max / norm_mean (abs error of the normalised map, the
    FP64 rows normalised with the GPU map's min/max over the masked interior)
    and raw_max / raw_mean (relative error of the raw map value, independent
    of any normalisation)."""
    j_means, j_stds = oracle.local_stats(img, bw, bh)
    mask, thr, nv = oracle.relevance_mask(img, bw, bh, j_stds, c)
    num, den = oracle.global_sums_f64(metric, img, bw, bh, j_stds, nv, thr, rows)
    npx = float(oracle.n_pixels(mask, bw // 2, bh // 2))
    raw = num / (den * npx + 1e-7)
    m = mask.ravel()[rows] > 0
    if metric in ("NRMSE", "Abs. diff. of StdDevs"):
        raw = np.where(m, np.where(raw == 0, 1.0, 1.0 / np.where(raw == 0, 1.0, raw)), raw)
    if c > 0:
        raw = raw * mask.ravel()[rows]
    out_raw, _ = clutils.global_map_host(metric, img, bw, bh, c, False, ctx=ctx)
    full = out_raw.ravel()
    sel = mask.ravel() > 0
    mn, mx = float(full[sel].min()), float(full[sel].max())
    exp_n = np.where(m, (raw - mn) / (mx - mn + 1e-7), raw)
    dn = np.abs(out.ravel()[rows] - exp_n)
    rel = (np.abs(full[rows] - raw) / np.maximum(np.abs(raw), 1e-30))[m]
    return {"norm_max": float(dn.max()), "norm_mean": float(dn.mean()),
            "raw_max": float(rel.max()) if rel.size else 0.0, "raw_mean": float(rel.mean()) if rel.size else 0.0,
            "rows": int(rows.size)}


def _rows(W, H, r, n, seed):
    """n distinct seeded interior pixels (raster indices)."""
    rng = np.random.default_rng(seed)
    idx = rng.choice((W - 2 * r) * (H - 2 * r), size=n, replace=False)
    ys, xs = np.divmod(idx, W - 2 * r)
    return ((ys + r) * W + xs + r).astype(np.int32)


@pytest.mark.parametrize("engine", ENGINES)
def test_global_256_pearson_sampled(ctx, engine):
    """256x256, 5x5, Pearson, relevance 0 (the reference's CPU-runnable case)."""
    img = synth.normalize_input(synth.image_256_spots(seed=0))
    ctx.set_engine(engine)
    out, info = clutils.global_map_host("Pearson's R", img, 5, 5, 0.0, True, ctx=ctx)
    e = _sampled_errors(ctx, out, info, img, "Pearson's R", 5, 5, 0.0, _rows(256, 256, 2, 4096, 1))
    _note(test="global_256_sampled", engine=engine, **e, info=info)
    assert e["norm_max"] <= GLOBAL_TOL[engine] and e["raw_max"] <= RAW_TOL[engine], e


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("metric", ["Pearson's R", "SSIM", "NRMSE"])
def test_global_1024_sampled(ctx, engine, metric):
    """1024x1024, 9x9 (K=49), relevance 1.0: 4096 sampled rows, each against
    every relevant block, against FP64."""
    img = synth.normalize_input(synth.image_1024_spots_random(seed=0))
    ctx.set_engine(engine)
    out, info = clutils.global_map_host(metric, img, 9, 9, 1.0, True, ctx=ctx)
    e = _sampled_errors(ctx, out, info, img, metric, 9, 9, 1.0, _rows(1024, 1024, 4, 4096, 2))
    _note(test="global_1024_sampled", engine=engine, metric=metric, **e, info=info)
    assert e["norm_max"] <= GLOBAL_TOL[engine] and e["raw_max"] <= RAW_TOL[engine], e


def test_global_2048_11x11_sampled(ctx):
    """2048x2048 elongated-spot image, 11x11 (K=81, K'=256: the tensor-core
    engine's 128-column tiles), Pearson with the relevance mask: 4096 sampled
    rows against FP64."""
    img = synth.normalize_input(synth.image_2048_elongated(seed=0))
    ctx.set_engine("tc")
    out, info = clutils.global_map_host("Pearson's R", img, 11, 11, 1.0, True, ctx=ctx)
    e = _sampled_errors(ctx, out, info, img, "Pearson's R", 11, 11, 1.0, _rows(2048, 2048, 5, 4096, 3))
    _note(test="global_2048_11x11_sampled", engine="tc", **e, info=info)
    assert info["k"] == 81 and info["n_relevant"] > 1_000_000
    assert e["norm_max"] <= GLOBAL_TOL["tc"] and e["raw_max"] <= RAW_TOL["tc"], e
