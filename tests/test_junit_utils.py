"""Host-side helpers pinned by the reference's own JUnit vectors
(tests/golden/reference_junit.json, extracted by tests/golden/make_golden.py):

* Utils.getReferenceBlock2D (src/test/java/UtilsTest.java
  GetReferenceBlock2DTest): a 5x5 block gives radius 2 x 2, mean 0.5 and std
  0.64549720 within 1e-6; a block with even dimensions gives null (None);
* Utils.getInputImage2D (GetInputImage2DTest, GetInputImage2DTestOverloaded):
  without normalisation the pixels come back unchanged; with it, 10..40 maps
  to 0, 1/3, 2/3, 1 within 1e-4.

Both the library mirror (sred_b200.utils over the C ABI) and the oracle's
restatement are checked.
"""
import json
from pathlib import Path

import numpy as np

import oracle
from sred_b200 import utils

J = json.loads((Path(__file__).resolve().parent / "golden" / "reference_junit.json").read_text())


def test_reference_block_2d_junit():
    v = J["reference_block_2d"]
    blk = np.asarray(v["pixels"], np.float32).reshape(v["height"], v["width"])
    rb = utils.get_reference_block_2d(blk)
    assert rb is not None
    assert (rb.width, rb.height) == (v["width"], v["height"])
    assert [rb.radius_width, rb.radius_height] == v["expected_radius"]
    assert rb.size > 0
    assert abs(rb.mean - v["expected_mean"]) <= v["tolerance"]
    assert abs(rb.std - v["expected_std"]) <= v["tolerance"]
    px, m, s = oracle.reference_block(blk)
    assert abs(m - v["expected_mean"]) <= v["tolerance"] and abs(s - v["expected_std"]) <= v["tolerance"]
    assert np.array_equal(rb.pixels[:rb.size], px)


def test_reference_block_2d_even_dimensions_is_none():
    v = J["reference_block_2d"]
    even = np.asarray(v["even_pixels"], np.float32).reshape(v["even_height"], v["even_width"])
    assert utils.get_reference_block_2d(even) is None


def test_input_image_2d_junit():
    v = J["input_image_2d"]
    p = v["plain"]
    px = np.asarray(p["pixels"], np.float32).reshape(p["height"], p["width"])
    r = utils.get_input_image_2d(px, normalize_output=False)
    assert (r.width, r.height, r.size) == (p["width"], p["height"], p["width"] * p["height"])
    assert np.array_equal(np.asarray(r.image_array, np.float32).ravel(), px.ravel())
    n = v["normalized"]
    px = np.asarray(n["pixels"], np.float32).reshape(n["height"], n["width"])
    r = utils.get_input_image_2d(px, normalize_output=True)
    assert (r.width, r.height, r.size) == (n["width"], n["height"], n["width"] * n["height"])
    got = np.asarray(r.image_array, np.float32).ravel()
    assert np.max(np.abs(got - np.asarray(n["expected"], np.float32))) <= n["tolerance"]
    assert np.array_equal(got, oracle.normalize_input(px).ravel())
