"""Host-side steps of the commands that need no GPU.

roi_offset_and_sigma restates VarianceStabilisingTransform2D_.meanAndStdDev
(java/VarianceStabilisingTransform2D_.java:116-133); checked here against the
same loop written out literally, value by value.
"""
import math

import numpy as np

from sred_b200 import plugins


def _java_mean_std(img, x, y, w, h):
    vals = [float(img[j, i]) for j in range(y, y + h) for i in range(x, x + w)]
    if not vals:
        return 0.0, 0.0
    s = sq = 0.0
    for v in vals:
        s += v
        sq += v * v
    mean = s / len(vals)
    var = sq / len(vals) - mean * mean
    return mean, (math.sqrt(var) if var >= 0 else math.nan)


def test_roi_offset_and_sigma_matches_the_java_loop():
    rng = np.random.default_rng(3)
    img = (rng.poisson(40.0, (60, 70)) * 2.0 + 100.0 + rng.normal(0, 5, (60, 70))).astype(np.float32)
    for roi in [(0, 0, 70, 60), (5, 7, 13, 9), (69, 59, 1, 1), (10, 10, 0, 5)]:
        got = plugins.roi_offset_and_sigma(img, roi)
        exp = _java_mean_std(img, *roi)
        assert got[0] == exp[0]
        assert got[1] == exp[1] or (math.isnan(got[1]) and math.isnan(exp[1]))
    # a constant ROI: the one-pass variance may round below zero (NaN) or to 0, as in Java
    flat = np.full((8, 8), 0.1, np.float32)
    got, exp = plugins.roi_offset_and_sigma(flat, (0, 0, 8, 8)), _java_mean_std(flat, 0, 0, 8, 8)
    assert got[0] == exp[0] and (got[1] == exp[1] or (math.isnan(got[1]) and math.isnan(exp[1])))


def test_output_buffers_are_checked_before_any_call():
    """The host-buffer entry points refuse an `out` they could not fill in
    place (wrong dtype, strided, wrong size) before touching the library."""
    import pytest
    from sred_b200 import clutils
    good = np.zeros((4, 5), np.float32)
    assert clutils._out_buffer(good, 20, "x").base is good
    for bad in (np.zeros((4, 5), np.float64), np.zeros((4, 10), np.float32)[:, ::2], np.zeros(21, np.float32)):
        with pytest.raises(ValueError):
            clutils._out_buffer(bad, 20, "x")
