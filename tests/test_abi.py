"""The C-ABI library loads, exports what include/sred.h declares, and its
host-only entry points agree with the oracle. No GPU needed."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from sred_b200 import _lib, utils

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "sred.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sred_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    decl = declared_symbols()
    assert len(decl) >= 16
    for s in decl:
        assert hasattr(L, s), s
    assert sorted(_lib.EXPORTS) == decl


def test_status_strings():
    assert _lib.status_string(0) == "ok"
    assert "metric" in _lib.status_string(_lib.ERR_UNKNOWN_METRIC)


def test_block_size_matches_oracle():
    for bw in range(3, 22, 2):
        for bh in range(3, 22, 2):
            assert utils.block_size(bw, bh) == oracle.block_size(bw, bh)


def test_create_without_device_reports_nodev():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(_lib.SredError) as ei:
        _lib.Context(0)
    assert ei.value.status == _lib.ERR_NODEV


@pytest.mark.parametrize("shape", [(3, 3), (5, 5), (7, 5), (15, 15)])
def test_reference_block_matches_oracle(shape):
    rng = np.random.default_rng(sum(shape))
    blk = rng.uniform(0, 1, shape).astype(np.float32)
    a = utils.get_reference_block_2d(blk)
    px, m, s = oracle.reference_block(blk)
    assert a.size == px.size
    assert np.array_equal(a.pixels, px) and a.mean == m and a.std == s
    assert utils.get_reference_block_2d(np.zeros((4, 5), np.float32)) is None


def test_normalize_image_golden(junit):
    g = junit["normalize_image_2d"]
    out = utils.normalize_image_2d(np.array(g["image"], np.float32), 4, 4, g["border_width"],
                                   g["border_height"], np.array(g["mask"], np.float32))
    np.testing.assert_allclose(out, g["expected"], atol=g["tolerance"])
    g = junit["normalize_image_2d_invalid"]
    with pytest.raises(ValueError):
        utils.normalize_image_2d(np.array(g["image"], np.float32), 4, 4, 0, 0, np.array(g["mask"], np.float32))


def test_apply_mask_golden(junit):
    g = junit["apply_mask_2d"]
    a = np.array(g["image"], np.float32)
    out = utils.apply_mask_2d(a, 3, 3, np.array(g["mask"], np.float32))
    assert np.array_equal(out, np.array(g["expected"], np.float32))


def test_header_cites_reference_for_each_entry_point():
    text = (ROOT / "include" / "sred.h").read_text()
    for fn in ["sred_local_statistics_2d", "sred_mean_noise_var_2d", "sred_relevance_mask_2d",
               "sred_calculate_global_repetition_map_2d", "sred_calculate_block_repetition_map_2d",
               "sred_reference_block_2d", "sred_normalize_image_2d", "sred_patch_hu_map_2d",
               "sred_hu_map_2d", "sred_phase_correlation_map_2d"]:
        i = text.index(fn + "(")
        comment = text[text.rindex("/*", 0, i):i]
        assert "java/" in comment or "cl/" in comment, fn
