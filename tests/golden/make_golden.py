"""Regenerate the golden fixtures in this folder.

Two kinds of fixtures are written:

1. ``reference_junit.json``: the known-answer vectors of the reference's own
   JUnit tests, read as text from a SReD checkout
   (``src/test/java/CLUtilsTest.java`` and ``src/test/java/UtilsTest.java``):
   inputs, parameters and expected outputs of the local-statistics,
   block-map, relevance-mask, normalisation and mask tests.

2. ``global_refshim.npz``: outputs of the reference's own global-map and
   block-map kernels (compiled for the CPU by ``oracle/refshim/build.py``) on
   small seeded synthetic images, with the Java host steps applied by the
   oracle. No reference test pins the global map; these frozen outputs do.

3. ``shape_refshim.npz``: outputs of the reference's shape-metric kernels
   (``cl/kernelGetPatchHu2D.cl``, ``cl/kernelGetHuMap.cl`` and, with the
   repairs listed in ``oracle/refshim/build.py``,
   ``cl/kernelGetPhaseCorrelationMap.cl``), compiled the same way, on small
   seeded images. No reference test covers these kernels.

4. ``volume_refshim.npz``: outputs of the reference's 3D local-statistics and
   3D block-map kernels (``cl/kernelGetLocalStatistics3D.cl``,
   ``cl/kernelGetBlock{Pearson,Ssim,Nrmse,AbsDiffStds}3D.cl``), compiled the
   same way, on small seeded volumes, with the Java host steps of
   ``getBlock*3D`` applied by the oracle; and for three of the volumes the
   3D global maps of ``cl/kernelGetGlobal*3D.cl`` (with the two repairs listed
   in ``oracle/refshim/build.py``) with the host steps of ``getGlobal*3D``.
   No reference test covers 3D.

5. ``relevance_refshim.npz``: outputs of the relevance-mask tools' kernels
   (``cl/kernelGetRelevanceMask2D.cl``, the local variance, and
   ``cl/kernelGetLocalMeans.cl``, the local std) on small seeded images.

Usage: ``python tests/golden/make_golden.py [--reference <SReD checkout>] [--only volume ...]``
(default: $SRED_REFERENCE, as ``oracle/refshim/build.py``)
"""
from __future__ import annotations

import argparse
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
from sred_b200 import synth  # noqa: E402

FLOAT = r"[-+]?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?f?"


def _method(src: str, name: str) -> str:
    i = src.index(f"void {name}(")
    depth, j, started = 0, src.index("{", i), False
    for k in range(j, len(src)):
        if src[k] == "{":
            depth += 1
            started = True
        elif src[k] == "}":
            depth -= 1
            if started and depth == 0:
                return src[j:k + 1]
    raise ValueError(name)


def _array(body: str, var: str) -> list[float]:
    m = re.search(r"\b" + re.escape(var) + r"\s*=\s*(?:new\s+float\s*\[\s*\]\s*)?\{([^}]*)\}", body)
    if not m:
        raise ValueError(var)
    return [float(t.rstrip("f")) for t in re.findall(FLOAT, m.group(1))]


def _scalar(body: str, pattern: str) -> float:
    m = re.search(pattern, body)
    if not m:
        raise ValueError(pattern)
    return float(m.group(1).rstrip("f"))


def _class(src: str, name: str) -> str:
    """Body of the (nested) class `name`."""
    i = src.index(f"class {name}")
    j = src.index("{", i)
    depth = 0
    for k in range(j, len(src)):
        depth += src[k] == "{"
        depth -= src[k] == "}"
        if depth == 0:
            return src[j:k + 1]
    raise ValueError(name)


def junit_vectors(ref: Path) -> dict:
    cl = (ref / "src/test/java/CLUtilsTest.java").read_text()
    ut = (ref / "src/test/java/UtilsTest.java").read_text()
    out: dict = {"source": "SReD src/test/java (JUnit 5)"}

    b = _method(cl, "testGetLocalStatistics2D")
    out["local_statistics_2d"] = {
        "cite": "src/test/java/CLUtilsTest.java testGetLocalStatistics2D",
        "width": 5, "height": 5, "block_width": 3, "block_height": 3,
        "image": _array(b, "inputImageData"),
        "expected_means": _array(b, "expectedLocalMeans"),
        "expected_stds": _array(b, "expectedLocalStds"),
        "tolerance": 1e-7,
    }
    tol = {"testGetBlockPearson2D": 1e-6, "testGetBlockSsim2D": 1e-7,
           "testGetBlockNrmse2D": 1e-5, "testGetBlockAbsDiffStds2D": 1e-7}
    metric = {"testGetBlockPearson2D": "Pearson's R", "testGetBlockSsim2D": "SSIM",
              "testGetBlockNrmse2D": "NRMSE (inverted)",
              "testGetBlockAbsDiffStds2D": "Abs. Diff. of StdDevs."}
    out["block_maps_2d"] = []
    for name in tol:
        b = _method(cl, name)
        out["block_maps_2d"].append({
            "cite": f"src/test/java/CLUtilsTest.java {name}",
            "metric": metric[name], "width": 10, "height": 10, "block_width": 3,
            "block_height": 3, "relevance_constant": 0.0, "normalize": True,
            "image": _array(b, "imageArray"), "block": _array(b, "block"),
            "expected": _array(b, "expectedResult"), "tolerance": tol[name],
        })
    b = _method(ut, "GetRelevanceMaskTest")
    out["relevance_mask"] = {
        "cite": "src/test/java/UtilsTest.java GetRelevanceMaskTest",
        "width": 50, "height": 50, "java_random_seed": 42,
        "block_radius_width": 2, "block_radius_height": 2,
        "relevance_constant": _scalar(b, r"float relevanceConstant\s*=\s*(" + FLOAT + ")"),
        "expected_threshold": _scalar(b, r"assertEquals\((" + FLOAT + r"),\s*relevanceMask\.getRelevanceThreshold"),
        "expected_noise_var": _scalar(b, r"assertEquals\((" + FLOAT + r"),\s*relevanceMask\.getNoiseMeanVariance"),
    }
    b = _method(ut, "testNormalizeImageWithBinaryMask")
    out["normalize_image_2d"] = {
        "cite": "src/test/java/UtilsTest.java testNormalizeImageWithBinaryMask",
        "width": 4, "height": 4, "border_width": 1, "border_height": 1,
        "image": _array(b, "imageArray"), "mask": _array(b, "mask"),
        "expected": _array(b, "expectedArray"), "tolerance": 1e-4,
    }
    b = _method(ut, "testNormalizeImageWithInvalidMask")
    out["normalize_image_2d_invalid"] = {
        "cite": "src/test/java/UtilsTest.java testNormalizeImageWithInvalidMask",
        "width": 4, "height": 4, "image": _array(b, "imageArray"), "mask": _array(b, "invalidMask"),
    }
    c = _class(ut, "GetReferenceBlock2DTest")
    valid = _method(c, "testGetReferenceBlock2DValidBlock")
    out["reference_block_2d"] = {
        "cite": "src/test/java/UtilsTest.java GetReferenceBlock2DTest",
        "width": 5, "height": 5, "pixels": _array(_method(c, "setup"), "pixels"),
        "expected_mean": _scalar(valid, r"assertEquals\((" + FLOAT + r"),\s*block\.getMean\(\)"),
        "expected_std": _scalar(valid, r"assertEquals\((" + FLOAT + r"),\s*block\.getStd\(\)"),
        "expected_radius": [2, 2], "tolerance": 1e-6,
        "even_pixels": _array(_method(c, "testGetReferenceBlock2DEvenDimensions"), "evenPixels"),
        "even_width": 4, "even_height": 4,
    }
    c = _class(ut, "GetInputImage2DTestOverloaded")
    nn = _method(c, "testGetInputImage2D_NoStabilization_NoNormalization")
    wn = _method(c, "testGetInputImage2D_WithNormalization")
    out["input_image_2d"] = {
        "cite": "src/test/java/UtilsTest.java GetInputImage2DTest, GetInputImage2DTestOverloaded",
        "plain": {"width": 3, "height": 3, "pixels": _array(nn, "pixels")},
        "normalized": {"width": 2, "height": 2, "pixels": _array(wn, "pixels"),
                       "expected": _array(wn, "normalizedPixels"), "tolerance": 1e-4},
    }
    b = _method(ut, "testApplyMask2D")
    out["apply_mask_2d"] = {
        "cite": "src/test/java/UtilsTest.java testApplyMask2D",
        "image": _array(b, "imageArray"), "mask": _array(b, "mask"),
        "expected": _array(b, "expectedResult"),
    }
    return out


GLOBAL_CASES = [
    # (name, W, H, lattice, seed, bw, bh, relevance constants)
    ("spots48x40_3x3", 48, 40, 4, 11, 3, 3, (0.0, 1.0)),
    ("spots40x44_5x5", 40, 44, 4, 12, 5, 5, (0.0, 1.0)),
    ("spots52x36_5x3", 52, 36, 5, 13, 5, 3, (0.0, 2.0)),
    ("spots36x36_9x9", 36, 36, 3, 14, 9, 9, (0.0,)),
]


def flat_image() -> np.ndarray:
    """Image with exactly flat regions (exercises the sigma == 0 special cases)."""
    img = np.zeros((32, 40), np.float32)
    img[8:20, 10:30] = 0.5
    img[22:28, 4:12] = 1.0
    rng = np.random.default_rng(5)
    img[0:6, :] = rng.uniform(0, 1, (6, 40)).astype(np.float32)
    return img


def refshim_fixtures() -> dict:
    if oracle.refshim() is None:
        raise SystemExit("refshim not built; run oracle/refshim/build.py with a reference checkout")
    fx: dict = {}
    images = {name: synth.normalize_input(synth.spot_image(W, H, lat, seed=seed))
              for name, W, H, lat, seed, *_ in GLOBAL_CASES}
    images["flat32x40_3x3"] = flat_image()
    cases = [(n, bw, bh, cs) for n, _, _, _, _, bw, bh, cs in GLOBAL_CASES]
    cases.append(("flat32x40_3x3", 3, 3, (0.0,)))
    for name, bw, bh, cs in cases:
        img = images[name]
        fx[f"{name}/image"] = img
        for c in cs:
            for metric in oracle.GLOBAL_METRICS:
                r = oracle.global_map(metric, img, bw, bh, c, normalize=True, use_refshim=True)
                tag = f"{name}/c{c:g}/{metric}"
                fx[f"{tag}/num"] = r["num"]
                fx[f"{tag}/den"] = r["den"]
                fx[f"{tag}/map"] = r["map"]
            fx[f"{name}/c{c:g}/threshold"] = np.float32(r["threshold"])
            fx[f"{name}/c{c:g}/noise_var"] = np.float32(r["noise_var"])
        # block map against a block cut from the image itself
        K = oracle.block_size(bw, bh)
        y0, x0 = img.shape[0] // 2 - bh // 2, img.shape[1] // 3 - bw // 2
        px, bm, bs = oracle.reference_block(img[y0:y0 + bh, x0:x0 + bw])
        assert px.size == K
        fx[f"{name}/block/pixels"] = px
        fx[f"{name}/block/mean_std"] = np.array([bm, bs], np.float32)
        for metric in oracle.BLOCK_METRICS:
            for c in (0.0, 1.0):
                r = oracle.block_map(metric, img, px, bw, bh, bm, bs, c, True, use_refshim=True)
                fx[f"{name}/block/c{c:g}/{metric}/raw"] = r["raw"]
                fx[f"{name}/block/c{c:g}/{metric}/map"] = r["map"]
    return fx


SHAPE_CASES = [
    # (name, W, H, lattice, seed, bw, bh, phase): the phase kernel's CPU cost
    # grows with (W H)^2 (bw bh)^2, so it runs on the smaller cases only
    ("spots32x28_3x3", 32, 28, 4, 21, 3, 3, True),
    ("spots30x26_5x3", 30, 26, 5, 22, 5, 3, True),
    ("spots40x36_5x5", 40, 36, 4, 23, 5, 5, False),
    ("spots44x40_9x9", 44, 40, 3, 24, 9, 9, False),
]


def shape_fixtures() -> dict:
    fx: dict = {}
    cases = [(n, synth.normalize_input(synth.spot_image(W, H, lat, seed=seed)), bw, bh, ph)
             for n, W, H, lat, seed, bw, bh, ph in SHAPE_CASES]
    cases.append(("flat32x40_3x3", flat_image(), 3, 3, True))
    for name, img, bw, bh, phase in cases:
        fx[f"{name}/image"] = img
        means, stds = oracle.local_stats(img, bw, bh)
        y0, x0 = img.shape[0] // 2 - bh // 2, img.shape[1] // 3 - bw // 2
        px, bm, bs = oracle.reference_block(img[y0:y0 + bh, x0:x0 + bw])
        patch = oracle.hu_prepare_patch(px, bw, bh)
        fx[f"{name}/block/pixels"] = px
        fx[f"{name}/block/mean_std"] = np.array([bm, bs], np.float32)
        fx[f"{name}/patch_hu/patch"] = patch
        fx[f"{name}/patch_hu/map"] = oracle.patch_hu_map(patch, img, bw, bh, use_refshim=True)
        fx[f"{name}/hu_map"] = oracle.hu_map(img, bw, bh, means, stds, use_refshim=True).astype(np.float32)
        if phase:
            fx[f"{name}/phase_map"] = oracle.phase_map(img, bw, bh, means, stds,
                                                       use_refshim=True).astype(np.float32)
    return fx


VOLUME_CASES = [
    # (name, W, H, D, lattice, lattice_z, seed, bw, bh, bd)
    ("spots28x24x12_3x3x3", 28, 24, 12, 4, 2, 31, 3, 3, 3),
    ("spots30x26x14_5x3x3", 30, 26, 14, 4, 2, 32, 5, 3, 3),
    ("spots24x24x16_5x5x5", 24, 24, 16, 3, 2, 33, 5, 5, 5),
    ("spots26x22x12_7x5x3", 26, 22, 12, 3, 2, 34, 7, 5, 3),
]


# cases whose 3D global maps (the reference's 3D global kernels with their two
# repairs, see oracle/refshim/build.py) are frozen too
GLOBAL_VOLUME_CASES = ("spots28x24x12_3x3x3", "spots24x24x16_5x5x5", "flat24x20x10_3x3x3")


def flat_volume() -> np.ndarray:
    """Volume with exactly flat regions (the std == 0 special cases)."""
    v = np.zeros((10, 20, 24), np.float32)
    v[2:8, 4:14, 5:20] = 0.5
    v[:, 15:19, 2:8] = 1.0
    rng = np.random.default_rng(7)
    v[:, 0:3, :] = rng.uniform(0, 1, (10, 3, 24)).astype(np.float32)
    return v


def volume_fixtures() -> dict:
    fx: dict = {}
    cases = [(n, synth.normalize_input(synth.spot_volume(W, H, D, lat, latz, seed=seed)), bw, bh, bd)
             for n, W, H, D, lat, latz, seed, bw, bh, bd in VOLUME_CASES]
    cases.append(("flat24x20x10_3x3x3", flat_volume(), 3, 3, 3))
    for name, vol, bw, bh, bd in cases:
        fx[f"{name}/volume"] = vol
        means, stds = oracle.local_stats3d(vol, bw, bh, bd, use_refshim=True)
        fx[f"{name}/means"] = means
        fx[f"{name}/stds"] = stds
        D, H, W = vol.shape
        z0, y0, x0 = D // 2 - bd // 2, H // 2 - bh // 2, W // 3 - bw // 2
        px, bm, bs = oracle.reference_block3d(vol[z0:z0 + bd, y0:y0 + bh, x0:x0 + bw])
        assert px.size == oracle.block_size3d(bw, bh, bd)
        fx[f"{name}/block/pixels"] = px
        fx[f"{name}/block/mean_std"] = np.array([bm, bs], np.float32)
        for c in (0.0, 1.0):
            mask, nv = oracle.relevance_mask3d(stds, bw, bh, bd, c)
            fx[f"{name}/c{c:g}/mask"] = mask
            fx[f"{name}/c{c:g}/noise_var"] = nv
            for metric in oracle.BLOCK_METRICS_3D:
                r = oracle.block_map3d(metric, vol, px, bw, bh, bd, bm, bs, c, True, use_refshim=True)
                fx[f"{name}/{metric}/raw"] = r["raw"]  # the kernel's output does not depend on c
                fx[f"{name}/c{c:g}/{metric}/map"] = r["map"]
        if name in GLOBAL_VOLUME_CASES:
            for c in (0.0, 1.0):
                for metric in oracle.GLOBAL_METRICS:
                    g = oracle.global_map3d(metric, vol, bw, bh, bd, c, True, use_refshim=True)
                    fx[f"{name}/global/c{c:g}/{metric}/map"] = g["map"]
                fx[f"{name}/global/c{c:g}/n_pixels"] = g["n_pixels"]
    return fx


RELEVANCE_CASES = [
    # (name, W, H, lattice, seed, block)
    ("spots60x50_3x3", 60, 50, 5, 41, 3),
    ("spots72x64_5x5", 72, 64, 6, 42, 5),
    ("spots48x56_7x7", 48, 56, 4, 43, 7),
]


def relevance_fixtures() -> dict:
    fx: dict = {}
    for name, W, H, lat, seed, b in RELEVANCE_CASES:
        img = synth.normalize_input(synth.spot_image(W, H, lat, seed=seed))
        fx[f"{name}/image"] = img
        fx[f"{name}/var"] = oracle.local_var2d(img, b, b, 0, use_refshim=True)
        fx[f"{name}/std"] = oracle.local_var2d(img, b, b, 1, use_refshim=True)
    return fx


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    sys.path.insert(0, str(HERE.parent.parent / "oracle" / "refshim"))
    from build import reference_root  # noqa: E402
    ap.add_argument("--reference", default=str(reference_root()))
    ap.add_argument("--only", choices=["junit", "global", "shape", "volume", "relevance"], action="append",
                    help="regenerate only these fixture files (default: all)")
    a = ap.parse_args(argv)
    only = set(a.only or ["junit", "global", "shape", "volume", "relevance"])
    if "junit" in only:
        vec = junit_vectors(Path(a.reference))
        (HERE / "reference_junit.json").write_text(json.dumps(vec, indent=1))
        print("wrote", HERE / "reference_junit.json")
    for kind, fname, make in (("global", "global_refshim.npz", refshim_fixtures),
                              ("shape", "shape_refshim.npz", shape_fixtures),
                              ("volume", "volume_refshim.npz", volume_fixtures),
                              ("relevance", "relevance_refshim.npz", relevance_fixtures)):
        if kind in only:
            fx = make()
            np.savez_compressed(HERE / fname, **fx)
            print("wrote", HERE / fname, len(fx), "arrays")
    return 0


if __name__ == "__main__":
    sys.exit(main())
