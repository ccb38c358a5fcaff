"""Failure detection, without faulting, trapping or hanging the GPU.

* Host-side injection: SRED_FAULT=alloc / launch makes the library report an
  allocation or launch failure (SRED_ERR_OOM / SRED_ERR_LAUNCH) before it
  touches the GPU for that step; the next call on the same context works and
  gives the same map. The reference's host turns such failures into a
  RuntimeException (java/CLUtils.java:175-180).
* Bounded device waits: every mbarrier wait of the tensor-core kernel gives up
  after a host-set limit. With a 0.2 s limit and the copy producer told to
  stop before its first tile's operands (so nothing is in flight), the waits
  run out, the kernel records the expiry and returns, the call reports
  SRED_ERR_TIMEOUT, and the next call on the same context gives the normal
  map.
"""
import ctypes as C
import os

import numpy as np
import pytest

from sred_b200 import _lib, clutils, synth, utils

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def img():
    return synth.normalize_input(synth.spot_image(96, 80, 6, seed=21))


@pytest.fixture()
def ctx():
    c = _lib.Context(0, "tc")
    yield c
    c.close()


def _map(ctx, img, metric="Pearson's R"):
    return clutils.global_map_host(metric, img, 5, 5, 1.0, True, ctx=ctx)[0]


@pytest.mark.parametrize("fault,status", [("alloc", _lib.ERR_OOM), ("launch", _lib.ERR_LAUNCH)])
def test_injected_host_failures_leave_the_context_usable(ctx, img, fault, status, monkeypatch):
    good = _map(ctx, img)
    monkeypatch.setenv("SRED_FAULT", fault)
    with pytest.raises(_lib.SredError) as ei:
        _map(ctx, img)
    assert ei.value.status == status
    ref = utils.get_reference_block_2d(img[10:15, 20:25])
    with pytest.raises(_lib.SredError) as ei:
        clutils.calculate_block_repetition_map_2d("Pearson's R", utils.InputImage2D(img.ravel(), 96, 80), ref, 0.0,
                                                  True, ctx=ctx)
    assert ei.value.status == status
    monkeypatch.delenv("SRED_FAULT")
    again = _map(ctx, img)
    np.testing.assert_allclose(again, good, rtol=0, atol=1e-6)


def test_tensor_core_wait_limit_expires_with_nothing_in_flight(ctx, img):
    L = ctx._L
    good = _map(ctx, img)
    ctx.check(L.sred_debug_set_tc_wait(ctx.h, 200_000_000, 0), "sred_debug_set_tc_wait")
    with pytest.raises(_lib.SredError) as ei:
        _map(ctx, img)
    assert ei.value.status == _lib.ERR_TIMEOUT
    # a tile index past the map's work: no effect
    ctx.check(L.sred_debug_set_tc_wait(ctx.h, 200_000_000, 1 << 40), "sred_debug_set_tc_wait")
    np.testing.assert_allclose(_map(ctx, img), good, rtol=0, atol=1e-6)
    ctx.check(L.sred_debug_set_tc_wait(ctx.h, 0, -1), "sred_debug_set_tc_wait")
    for metric in ("Pearson's R", "SSIM", "NRMSE"):
        out = _map(ctx, img, metric)
        assert np.isfinite(out).all()
    np.testing.assert_allclose(_map(ctx, img), good, rtol=0, atol=1e-6)
    assert L.sred_debug_set_tc_wait(ctx.h, 0, -2) == _lib.ERR_ARG
