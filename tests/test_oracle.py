"""Pin the CPU oracle before trusting it.

The FP32 restatement must reproduce (a) the reference's JUnit known-answer
vectors and (b) the reference's own kernels compiled for the CPU (frozen in
tests/golden/global_refshim.npz, and live when oracle/_ref is built), bit for
bit. The FP64 judge must agree with the FP32 path to FP32 accuracy.
"""
import numpy as np
import pytest

import oracle


def _ref_block_as_junit(block, bw, bh):
    """ReferenceBlock2D as the JUnit tests build it: raw ellipse pixels, FP32
    mean and (K-1) standard deviation (src/test/java/CLUtilsTest.java:560-600)."""
    f = np.float32
    rw, rh = bw // 2, bh // 2
    px = []
    for y in range(bh):
        for x in range(bw):
            dx, dy = f(x - rw), f(y - rh)
            if (dx * dx) / f(rw * rw) + (dy * dy) / f(rh * rh) <= f(1):
                px.append(f(block[y * bw + x]))
    px = np.array(px, np.float32)
    mean = f(0)
    for v in px:
        mean = f(mean + v)
    mean = f(mean / f(px.size))
    sd = f(0)
    for v in px:
        sd = f(sd + f(f(v - mean) * f(v - mean)))
    sd = f(sd / f(f(px.size) - f(1)))
    sd = f(np.sqrt(np.float64(sd)))
    return px, mean, sd


def test_block_size_ellipse():
    assert [oracle.block_size(b, b) for b in (3, 5, 7, 9, 11, 13, 15)] == [5, 13, 29, 49, 81, 113, 149]


def test_local_statistics_golden(junit):
    g = junit["local_statistics_2d"]
    img = np.array(g["image"], np.float32).reshape(g["height"], g["width"])
    m, s = oracle.local_stats(img, g["block_width"], g["block_height"])
    np.testing.assert_allclose(m.ravel(), g["expected_means"], atol=g["tolerance"], rtol=0)
    np.testing.assert_allclose(s.ravel(), g["expected_stds"], atol=g["tolerance"], rtol=0)


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("shim", [False, True])
def test_block_map_golden(junit, idx, shim):
    g = junit["block_maps_2d"][idx]
    if shim and oracle.refshim() is None:
        pytest.skip("refshim not built")
    img = np.array(g["image"], np.float32).reshape(g["height"], g["width"])
    px, mean, sd = _ref_block_as_junit(g["block"], g["block_width"], g["block_height"])
    r = oracle.block_map(g["metric"], img, px, g["block_width"], g["block_height"], mean, sd,
                         g["relevance_constant"], g["normalize"], use_refshim=shim)
    out = r["map"].ravel()
    assert np.all((out >= 0) & (out <= 1))
    np.testing.assert_allclose(out, g["expected"], atol=g["tolerance"], rtol=0)


def test_relevance_mask_golden(junit):
    g = junit["relevance_mask"]
    W, H = g["width"], g["height"]
    # Rebuild the test's inputs: java.util.Random(42), draws interleaved per pixel.
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
    img, stds = img.reshape(H, W), stds.reshape(H, W)
    bw, bh = 2 * g["block_radius_width"] + 1, 2 * g["block_radius_height"] + 1
    mask, thr, nv = oracle.relevance_mask(img, bw, bh, stds, g["relevance_constant"])
    assert thr == np.float32(g["expected_threshold"])
    assert float(nv) == g["expected_noise_var"]
    assert set(np.unique(mask)) <= {0.0, 1.0}


def test_normalize_golden(junit):
    g = junit["normalize_image_2d"]
    img = np.array(g["image"], np.float32).reshape(4, 4)
    mask = np.array(g["mask"], np.float32).reshape(4, 4)
    out = oracle.normalize_image(img, g["border_width"], g["border_height"], mask)
    np.testing.assert_allclose(out.ravel(), g["expected"], atol=g["tolerance"])
    g = junit["normalize_image_2d_invalid"]
    with pytest.raises(ValueError):
        oracle.normalize_image(np.array(g["image"], np.float32).reshape(4, 4), 0, 0,
                               np.array(g["mask"], np.float32).reshape(4, 4))


def _fixture_cases(fx):
    names = sorted({k.split("/")[0] for k in fx})
    for n in names:
        bw, bh = (int(v) for v in n.rsplit("_", 1)[1].split("x"))
        cs = sorted({k.split("/")[1] for k in fx if k.startswith(n + "/c")})
        for c in cs:
            yield n, bw, bh, float(c[1:])


def test_global_f32_matches_refshim_fixtures(refshim_fx):
    """Oracle port == the reference's own kernels (frozen), bit for bit."""
    fx = refshim_fx
    n_cases = 0
    for name, bw, bh, c in _fixture_cases(fx):
        img = fx[f"{name}/image"]
        for metric in oracle.GLOBAL_METRICS:
            r = oracle.global_map(metric, img, bw, bh, c, normalize=True)
            tag = f"{name}/c{c:g}/{metric}"
            assert np.array_equal(r["num"], fx[f"{tag}/num"]), tag
            assert np.array_equal(r["den"], fx[f"{tag}/den"]), tag
            assert np.array_equal(r["map"], fx[f"{tag}/map"], equal_nan=True), tag
            n_cases += 1
    assert n_cases >= 30


def test_block_f32_matches_refshim_fixtures(refshim_fx):
    fx = refshim_fx
    for name in sorted({k.split("/")[0] for k in fx}):
        bw, bh = (int(v) for v in name.rsplit("_", 1)[1].split("x"))
        img = fx[f"{name}/image"]
        px = fx[f"{name}/block/pixels"]
        bm, bs = fx[f"{name}/block/mean_std"]
        for metric in oracle.BLOCK_METRICS:
            for c in (0.0, 1.0):
                r = oracle.block_map(metric, img, px, bw, bh, bm, bs, c, True)
                tag = f"{name}/block/c{c:g}/{metric}"
                assert np.array_equal(r["raw"], fx[f"{tag}/raw"]), tag
                assert np.array_equal(r["map"], fx[f"{tag}/map"]), tag


@pytest.mark.skipif(oracle.refshim() is None, reason="refshim not built")
@pytest.mark.parametrize("metric", list(oracle.GLOBAL_METRICS))
def test_global_f32_matches_refshim_live(metric):
    from sred_b200 import synth
    img = synth.normalize_input(synth.spot_image(46, 38, 4, seed=99))
    for bw, bh in ((3, 5), (7, 7)):
        a = oracle.global_map(metric, img, bw, bh, 1.0)
        b = oracle.global_map(metric, img, bw, bh, 1.0, use_refshim=True)
        assert np.array_equal(a["num"], b["num"]) and np.array_equal(a["den"], b["den"])
        assert np.array_equal(a["map"], b["map"])


@pytest.mark.parametrize("metric", list(oracle.GLOBAL_METRICS))
def test_f64_judge_close_to_f32(refshim_fx, metric):
    img = refshim_fx["spots40x44_5x5/image"]
    a = oracle.global_map(metric, img, 5, 5, 1.0, precision="f32")
    b = oracle.global_map(metric, img, 5, 5, 1.0, precision="f64")
    m = a["mask"] > 0
    np.testing.assert_allclose(a["map"][m], b["map"][m], atol=2e-5, rtol=0)


# ---------------------------------------------------------------------------
# Shape metrics (cl/kernelGetPatchHu2D.cl, cl/kernelGetHuMap.cl,
# cl/kernelGetPhaseCorrelationMap.cl): the restatement against the
# reference's kernels, frozen in tests/golden/shape_refshim.npz
# ---------------------------------------------------------------------------

def _shape_cases(fx):
    for n in sorted({k.split("/")[0] for k in fx}):
        bw, bh = (int(v) for v in n.rsplit("_", 1)[1].split("x"))
        yield n, bw, bh


def test_patch_hu_matches_refshim_fixtures(shape_fx):
    fx = shape_fx
    for name, bw, bh in _shape_cases(fx):
        img = fx[f"{name}/image"]
        patch = oracle.hu_prepare_patch(fx[f"{name}/block/pixels"], bw, bh)
        assert np.array_equal(patch, fx[f"{name}/patch_hu/patch"]), name
        got = oracle.patch_hu_map(patch, img, bw, bh)
        assert np.array_equal(got, fx[f"{name}/patch_hu/map"], equal_nan=True), name


def test_hu_map_matches_refshim_fixtures(shape_fx):
    fx = shape_fx
    for name, bw, bh in _shape_cases(fx):
        got = oracle.hu_map(fx[f"{name}/image"], bw, bh).astype(np.float32)
        assert np.array_equal(got, fx[f"{name}/hu_map"]), name


def test_phase_map_matches_refshim_fixtures(shape_fx):
    fx = shape_fx
    n = 0
    for name, bw, bh in _shape_cases(fx):
        if f"{name}/phase_map" not in fx:
            continue
        got = oracle.phase_map(fx[f"{name}/image"], bw, bh).astype(np.float32)
        assert np.array_equal(got, fx[f"{name}/phase_map"]), name
        n += 1
    assert n >= 3


def test_shape_f64_judges_close_to_f32(shape_fx):
    """The FP64-accumulated judges agree with the FP32 reference order."""
    img = shape_fx["spots32x28_3x3/image"]
    for fn in (oracle.hu_map, oracle.phase_map):
        a = fn(img, 3, 3)
        b = fn(img, 3, 3, precision="f64")
        assert float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) < 2e-5


@pytest.mark.skipif(oracle.refshim() is None, reason="refshim not built")
def test_shape_matches_refshim_live():
    from sred_b200 import synth
    img = synth.normalize_input(synth.spot_image(26, 22, 4, seed=98))
    for bw, bh in ((3, 5), (7, 7)):
        patch = oracle.hu_prepare_patch(oracle.reference_block(img[5:5 + bh, 6:6 + bw])[0], bw, bh)
        assert np.array_equal(oracle.patch_hu_map(patch, img, bw, bh),
                              oracle.patch_hu_map(patch, img, bw, bh, use_refshim=True))
        assert np.array_equal(oracle.hu_map(img, bw, bh), oracle.hu_map(img, bw, bh, use_refshim=True))
    assert np.array_equal(oracle.phase_map(img, 3, 5), oracle.phase_map(img, 3, 5, use_refshim=True))


def test_block_phase_self_peak():
    """A block compared with itself peaks at displacement (0, 0): the
    1-based coordinates (1, 1) give sqrt(2)."""
    from sred_b200 import synth
    img = synth.normalize_input(synth.spot_image(30, 24, 4, seed=97))
    bw = bh = 5
    means, stds = oracle.local_stats(img, bw, bh)
    y, x = 11, 13
    # the block's own normalised ellipse pixels as the reference block
    K = oracle.block_size(bw, bh)
    blk = img[y - 2:y + 3, x - 2:x + 3]
    f = np.float32
    px = [blk[j, i] for j in range(5) for i in range(5)
          if (f(i - 2) ** 2) / f(4) + (f(j - 2) ** 2) / f(4) <= f(1)]
    px = np.array(px, np.float32) - means[y, x]
    assert px.size == K
    out = oracle.block_phase_raw(img, px, bw, bh, stds[y, x], means, stds)
    assert abs(out[y, x] - np.sqrt(2.0)) < 1e-6


def test_block_phase_matches_numpy_fft():
    """The block-map phase correlation (exact DFT) against numpy's FFT: the
    kernel's normalised cross-power spectrum of the two spectra (each / sqrt(n)),
    the real part of the inverse transform and the first strict maximum above 0
    in raster order, for every interior pixel and several block shapes."""
    from sred_b200 import synth
    eps = float(np.float32(1e-7))
    for bw, bh in [(5, 5), (9, 9), (15, 15), (7, 11), (13, 3)]:
        img = synth.normalize_input(synth.spot_image(34, 30, 4, seed=bw * 7 + bh))
        means, stds = oracle.local_stats(img, bw, bh)
        rw, rh = bw // 2, bh // 2
        f = np.float32
        ell = np.array([[(f(i - rw) ** 2) / f(rw * rw) + (f(j - rh) ** 2) / f(rh * rh) <= f(1) for i in range(bw)]
                        for j in range(bh)])
        y0, x0 = 15, 16
        ref_px = (img[y0 - rh:y0 + rh + 1, x0 - rw:x0 + rw + 1][ell] - means[y0, x0]).astype(np.float32)
        got = oracle.block_phase_raw(img, ref_px, bw, bh, stds[y0, x0], means, stds)
        R = np.zeros((bh, bw))
        R[ell] = ref_px.astype(np.float64) / (float(stds[y0, x0]) + eps)
        R = np.fft.fft2(R)
        sn = np.sqrt(bw * bh)
        for y in range(rh, img.shape[0] - rh):
            for x in range(rw, img.shape[1] - rw):
                P = np.zeros((bh, bw))
                blk = img[y - rh:y + rh + 1, x - rw:x + rw + 1].astype(np.float64)
                P[ell] = (blk[ell] - float(means[y, x])) / (float(stds[y, x]) + eps)
                F = np.fft.fft2(P) / sn
                m = R * np.conj(F)
                a, b = np.abs(m.real), np.abs(m.imag)
                X = (m.real * a + m.imag * b + 1j * (m.imag * a - m.real * b)) / (a * a + b * b + eps)
                v = np.real(np.fft.ifft2(X)) * (bw * bh) / sn
                pos = np.flatnonzero(v.ravel() > 0)
                if pos.size == 0:
                    exp = 0.0
                else:
                    k = pos[np.argmax(v.ravel()[pos])]
                    exp = float(np.float32(np.hypot(k % bw + 1, k // bw + 1)))
                assert got[y, x] == exp, (bw, bh, y, x)


# ---------------------------------------------------------------------------
# Variance stabilisation: the restatement against an independent numpy
# evaluation of java/VarianceStabilisingTransform2D_.java:136-151 and
# java/GATMinimizer2D.java (no reference test pins either)
# ---------------------------------------------------------------------------

def _poisson_gaussian(w, h, gain, sigma, offset, seed):
    """Poisson-Gaussian noise on an intensity that is constant over each cell
    of the objective's 6 x 6 block grid (20 to 500 photons per cell)."""
    rng = np.random.default_rng(seed)
    cells = rng.uniform(20, 500, (6, 6))
    lam = np.kron(cells, np.ones((h // 6, w // 6)))
    lam = np.pad(lam, ((0, h - lam.shape[0]), (0, w - lam.shape[1])), mode="edge")
    return (gain * rng.poisson(lam) + offset + rng.normal(0, sigma, (h, w))).astype(np.float32)


def test_gat_matches_numpy():
    img = _poisson_gaussian(60, 48, 2.0, 5.0, 100.0, 1)
    img[0, :5] = [-1e6, -50.0, 0.0, 1.0, 3.0]
    for g, s, o in [(2.0, 5.0, 100.0), (1.0, 10.0, 100.0), (0.5, 30.0, -20.0)]:
        c = 3.0 / 8.0 * g * g + s * s - g * o
        v = img.astype(np.float64)
        exp = np.where(g * v + c < 0, 0.0, (2.0 / g) * np.sqrt(np.maximum(g * v + c, 0))).astype(np.float32)
        assert np.array_equal(oracle.gat(img, g, s, o), exp)


def test_gat_objective_matches_numpy():
    img = _poisson_gaussian(66, 54, 2.0, 5.0, 100.0, 2)
    for g, s, o in [(2.0, 5.0, 100.0), (1.0, 10.0, 100.0)]:
        c = 3.0 / 8.0 * g * g + s * s - g * o
        v = img.astype(np.float64)
        t = np.where(v <= -c / g, 0.0, (2 / g) * np.sqrt(np.maximum(g * v + c, 0))).astype(np.float32)
        bw, bh = 66 // 6, 54 // 6
        err = 0.0
        for by in range(54 // bh):
            for bx in range(66 // bw):
                blk = t[by * bh:(by + 1) * bh, bx * bw:(bx + 1) * bw].astype(np.float64)
                sq = (t[by * bh:(by + 1) * bh, bx * bw:(bx + 1) * bw] ** 2).astype(np.float64)
                var = sq.sum() / blk.size - (blk.sum() / blk.size) ** 2
                err += (var - 1) ** 2 / 36
        assert abs(oracle.gat_objective(img, g, s, o) - err) <= 1e-9 * max(err, 1e-12)
    # the true parameters stabilise the variance much better than the reference's starting point
    assert oracle.gat_objective(img, 2.0, 5.0, 100.0) < 0.1 * oracle.gat_objective(img, 1.0, 10.0, 100.0)


# ---------------------------------------------------------------------------
# 3D block maps (cl/kernelGetLocalStatistics3D.cl,
# cl/kernelGetBlock*3D.cl and the host steps of java/CLUtils.java:1133-1637):
# the restatement against the reference's kernels, frozen in
# tests/golden/volume_refshim.npz
# ---------------------------------------------------------------------------

def volume_cases(fx):
    """(name, bw, bh, bd) of the cases in volume_refshim.npz."""
    for n in sorted({k.split("/")[0] for k in fx}):
        bw, bh, bd = (int(v) for v in n.rsplit("_", 1)[1].split("x"))
        yield n, bw, bh, bd


def test_block_size_ellipsoid():
    f = np.float32
    for bw, bh, bd in [(3, 3, 3), (5, 3, 7), (9, 9, 9), (11, 11, 11)]:
        rw, rh, rd = bw // 2, bh // 2, bd // 2
        k = 0
        for z in range(-rd, rd + 1):
            for y in range(-rh, rh + 1):
                for x in range(-rw, rw + 1):
                    k += (f(x * x) / f(rw * rw)) + (f(y * y) / f(rh * rh)) + (f(z * z) / f(rd * rd)) <= f(1)
        assert oracle.block_size3d(bw, bh, bd) == k


def test_volume_stats_match_refshim_fixtures(volume_fx):
    fx = volume_fx
    for name, bw, bh, bd in volume_cases(fx):
        m, s = oracle.local_stats3d(fx[f"{name}/volume"], bw, bh, bd)
        assert np.array_equal(m, fx[f"{name}/means"]) and np.array_equal(s, fx[f"{name}/stds"]), name


def test_volume_block_maps_match_refshim_fixtures(volume_fx):
    fx = volume_fx
    n = 0
    for name, bw, bh, bd in volume_cases(fx):
        vol = fx[f"{name}/volume"]
        px = fx[f"{name}/block/pixels"]
        bm, bs = fx[f"{name}/block/mean_std"]
        D, H, W = vol.shape
        z0, y0, x0 = D // 2 - bd // 2, H // 2 - bh // 2, W // 3 - bw // 2
        q = oracle.reference_block3d(vol[z0:z0 + bd, y0:y0 + bh, x0:x0 + bw])
        assert np.array_equal(q[0], px) and q[1] == bm and q[2] == bs, name
        for c in (0.0, 1.0):
            mask, nv = oracle.relevance_mask3d(fx[f"{name}/stds"], bw, bh, bd, c)
            assert np.array_equal(mask, fx[f"{name}/c{c:g}/mask"]) and nv == fx[f"{name}/c{c:g}/noise_var"]
            for metric in oracle.BLOCK_METRICS_3D:
                r = oracle.block_map3d(metric, vol, px, bw, bh, bd, bm, bs, c, True)
                assert np.array_equal(r["raw"], fx[f"{name}/{metric}/raw"]), (name, metric)
                assert np.array_equal(r["map"], fx[f"{name}/c{c:g}/{metric}/map"]), (name, c, metric)
                n += 1
    assert n == 40


def test_volume_flat_special_cases(volume_fx):
    """Flat blocks: Pearson and SSIM 1 where both stds are 0, 0 where one is."""
    fx = volume_fx
    name = "flat24x20x10_3x3x3"
    stds = fx[f"{name}/stds"]
    px, (bm, bs) = fx[f"{name}/block/pixels"], fx[f"{name}/block/mean_std"]
    flat = (stds == 0)
    flat[:1] = flat[-1:] = False
    flat[:, :1] = flat[:, -1:] = False
    flat[:, :, :1] = flat[:, :, -1:] = False
    assert flat.sum() > 100
    for metric in ("Pearson's R", "SSIM"):
        raw = fx[f"{name}/{metric}/raw"]
        assert np.all(raw[flat] == (1.0 if bs == 0 else 0.0))


@pytest.mark.skipif(oracle.refshim() is None, reason="refshim not built")
def test_volume_matches_refshim_live():
    from sred_b200 import synth
    vol = synth.normalize_input(synth.spot_volume(22, 20, 11, 3, 2, seed=77))
    for bw, bh, bd in ((3, 3, 5), (7, 3, 3), (5, 7, 5)):
        a = oracle.local_stats3d(vol, bw, bh, bd)
        b = oracle.local_stats3d(vol, bw, bh, bd, use_refshim=True)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        px, bm, bs = oracle.reference_block3d(vol[3:3 + bd, 5:5 + bh, 6:6 + bw])
        for metric in oracle.BLOCK_METRICS_3D:
            x = oracle.block_map3d(metric, vol, px, bw, bh, bd, bm, bs, 1.0)
            y = oracle.block_map3d(metric, vol, px, bw, bh, bd, bm, bs, 1.0, use_refshim=True)
            assert np.array_equal(x["raw"], y["raw"]) and np.array_equal(x["map"], y["map"]), metric


# 3D global maps: the restatement against the reference's 3D global kernels
# (two repairs, oracle/refshim/build.py), frozen in volume_refshim.npz

def test_global3d_f32_matches_refshim_fixtures(volume_fx):
    fx = volume_fx
    n = 0
    for name, bw, bh, bd in volume_cases(fx):
        if f"{name}/global/c0/Pearson's R/map" not in fx:
            continue
        vol = fx[f"{name}/volume"]
        for c in (0.0, 1.0):
            for metric in oracle.GLOBAL_METRICS:
                g = oracle.global_map3d(metric, vol, bw, bh, bd, c)
                assert np.array_equal(g["map"], fx[f"{name}/global/c{c:g}/{metric}/map"]), (name, c, metric)
                n += 1
            assert g["n_pixels"] == fx[f"{name}/global/c{c:g}/n_pixels"]
    assert n == 24


def test_global3d_f64_judge_close_to_f32(volume_fx):
    vol = volume_fx["spots28x24x12_3x3x3/volume"]
    for metric in oracle.GLOBAL_METRICS:
        for c in (0.0, 1.0):
            a = oracle.global_map3d(metric, vol, 3, 3, 3, c)["map"]
            b = oracle.global_map3d(metric, vol, 3, 3, 3, c, precision="f64")["map"]
            assert float(np.max(np.abs(a - b))) < 2e-5, (metric, c)


@pytest.mark.skipif(oracle.refshim() is None, reason="refshim not built")
def test_global3d_matches_refshim_live():
    from sred_b200 import synth
    vol = synth.normalize_input(synth.spot_volume(18, 16, 11, 3, 2, seed=78))
    for bw, bh, bd in ((3, 5, 3), (7, 3, 5)):
        means, stds = oracle.local_stats3d(vol, bw, bh, bd)
        mask, nv = oracle.relevance_mask3d(stds, bw, bh, bd, 0.5)
        thr = np.float32(nv * np.float32(0.5))
        for metric in oracle.GLOBAL_METRICS:
            a = oracle.global3d_sums_f32(metric, vol, bw, bh, bd, means, stds, nv, thr)
            b = oracle.global3d_sums_f32(metric, vol, bw, bh, bd, means, stds, nv, thr, use_refshim=True)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (bw, bh, bd, metric)


# Relevance-mask tools: the local variance / std of cl/kernelGetRelevanceMask2D.cl
# and cl/kernelGetLocalMeans.cl, frozen in relevance_refshim.npz

def test_tool_statistics_match_refshim_fixtures(relevance_fx):
    for name in sorted({k.split("/")[0] for k in relevance_fx}):
        b = int(name.rsplit("x", 1)[1])
        img = relevance_fx[f"{name}/image"]
        assert np.array_equal(oracle.local_var2d(img, b, b, 0), relevance_fx[f"{name}/var"]), name
        assert np.array_equal(oracle.local_var2d(img, b, b, 1), relevance_fx[f"{name}/std"]), name


@pytest.mark.skipif(oracle.refshim() is None, reason="refshim not built")
def test_tool_statistics_match_refshim_live():
    from sred_b200 import synth
    img = synth.normalize_input(synth.spot_image(45, 38, 4, seed=99))
    for b in (3, 5, 9):
        for ts in (0, 1):
            assert np.array_equal(oracle.local_var2d(img, b, b, ts), oracle.local_var2d(img, b, b, ts, True))


def test_tool_range_matches_mask_definition():
    """The literal loop of OptimiseRelevanceMask_: at all_zeros the mask is all
    0 and one step before it is not; at all_ones the interior is all 1."""
    from sred_b200 import synth
    img = synth.normalize_input(synth.spot_image(64, 48, 5, seed=7))
    v = oracle.local_var2d(img, 3, 3, 0)
    nv = oracle.tool_noise_var(img, 0)
    for step in (1.0, 0.05):
        ones, zeros = oracle.tool_range(v, 3, 3, nv, step)
        assert not oracle.tool_mask(v, 3, 3, nv, zeros).any()
        assert oracle.tool_mask(v, 3, 3, nv, np.float32(zeros - np.float32(step))).any()
        assert oracle.tool_mask(v, 3, 3, nv, ones)[1:-1, 1:-1].all()


def _poisson_gaussian3d(w, h, d, gain, sigma, offset, seed):
    """Poisson-Gaussian noise on an intensity constant over each cell of the
    3D objective's 6 x 6 x 6 block grid."""
    rng = np.random.default_rng(seed)
    cells = rng.uniform(20, 500, (6, 6, 6))
    lam = np.kron(cells, np.ones((d // 6, h // 6, w // 6)))
    lam = np.pad(lam, ((0, d - lam.shape[0]), (0, h - lam.shape[1]), (0, w - lam.shape[2])), mode="edge")
    return (gain * rng.poisson(lam) + offset + rng.normal(0, sigma, (d, h, w))).astype(np.float32)


def test_gat_objective3d_matches_numpy():
    vol = _poisson_gaussian3d(36, 30, 24, 2.0, 5.0, 100.0, 6)
    for g, s, o in [(2.0, 5.0, 100.0), (1.0, 10.0, 100.0)]:
        c = 3.0 / 8.0 * g * g + s * s - g * o
        v = vol.astype(np.float64)
        t = np.where(v <= -c / g, 0.0, (2 / g) * np.sqrt(np.maximum(g * v + c, 0))).astype(np.float32)
        blk = t.reshape(6, 4, 6, 5, 6, 6).astype(np.float64)  # bd=4, bh=5, bw=6
        var = (blk ** 2).mean(axis=(1, 3, 5)) - blk.mean(axis=(1, 3, 5)) ** 2
        err = float(((var - 1) ** 2).sum() / 216)
        assert abs(oracle.gat_objective3d(vol, g, s, o) - err) <= 1e-9 * err
    assert np.isnan(oracle.gat_objective3d(vol, 0.0, 1.0, 1.0))
    assert np.isnan(oracle.gat_objective3d(vol, 1.0, -1.0, 1.0))
    assert np.isnan(oracle.gat_objective3d(vol, 1.0, 1.0, -1.0))
    assert oracle.gat_objective3d(vol, 2.0, 5.0, 100.0) < 0.1 * oracle.gat_objective3d(vol, 1.0, 10.0, 100.0)


# Redundancy classification (java/ClassifyRedundancy_.java)

def test_java_random_generator():
    """The k-means generator is java.util.Random: its 48-bit sequence equals
    the one pinned by the reference's relevance-mask JUnit vectors (nextFloat =
    next(24) / 2^24, seed 42), and nextDouble follows the JDK's definition."""
    f = oracle.java_random_floats(42, 64)
    n24 = oracle.java_random_next(42, 24, 64)
    assert np.array_equal(f, (n24.astype(np.float64) / 2 ** 24).astype(np.float32))
    d = oracle.java_random_doubles(42, 8)
    # nextDouble draws next(26) then next(27) from consecutive states
    a26 = oracle.java_random_next(42, 26, 16).astype(np.int64)
    a27 = oracle.java_random_next(42, 27, 16).astype(np.int64)
    seq = [float(((int(a26[2 * i]) << 27) + int(a27[2 * i + 1])) * 2.0 ** -53) for i in range(8)]
    assert np.array_equal(d, np.array(seq))
    assert d[0] == 0.7275636800328681 and oracle.java_random_doubles(0, 1)[0] == 0.730967787376657
    assert 0.0 <= d.min() and d.max() < 1.0


def test_classify_redundancy_oracle_properties():
    from sred_b200 import synth
    m = synth.normalize_input(synth.spot_image(90, 70, 6, seed=3))
    for k in (1, 2, 4):
        out, kc, wcss = oracle.classify_redundancy(m, 2, k, seed=5)
        inner = out[2:-2, 2:-2].astype(int)
        counts = np.bincount(inner.ravel(), minlength=kc)
        assert kc == k and np.all(np.diff(counts) <= 0)  # ranked by size
        assert not out[:2].any() and not out[:, :2].any()
        # a Lloyd fixed point: each class is a contiguous value range
        vals = m[2:-2, 2:-2]
        cls = [vals[inner == j] for j in range(kc)]
        spans = sorted((c.min(), c.max()) for c in cls)
        assert all(spans[i][1] <= spans[i + 1][0] for i in range(len(spans) - 1))
        if k > 1:
            assert wcss < oracle.classify_redundancy(m, 2, 1, seed=5)[2]


def test_f_quantile_matches_scipy():
    """The Fisher test's threshold (QuadTree_.performFisherTest): F(df, df)
    quantiles by bisection of the regularised incomplete beta, in the oracle
    and in the library (host function), against scipy."""
    from scipy import stats
    from sred_b200 import _lib
    L = _lib.load()
    for df in [1, 2, 3, 8, 15, 63, 255, 4095, 65535, 1048575]:
        for p in [0.001, 0.01, 0.05, 0.5, 0.9]:
            e = stats.f.ppf(p, df, df)
            a = oracle.f_quantile(p, df)
            assert abs(a - e) <= 1e-10 * e, (df, p, a, e)
            assert L.sred_f_quantile(p, df) == a


def test_gat_tree_oracle_properties():
    from sred_b200 import synth
    rng = np.random.default_rng(1)
    lam = synth.spot_image(128, 96, 8, seed=2, read_noise=0.0).clip(0, None) / 4
    img = (2.0 * rng.poisson(lam) + 100 + rng.normal(0, 5.0, lam.shape)).astype(np.float32)
    r = oracle.gat_tree(img)
    b = r["boxes"]
    assert (b[:, 3] * b[:, 4]).sum() <= 128 * 96 and len(b) > 16  # disjoint leaves inside the image
    assert r["g0"] > 0 and np.isfinite(r["image"]).all()
