"""The tensor-core engine's work-item decode (global_tc.cu: decode_item,
compiled for the host from the library's own source) lists the same tiles in
the same order as the Python mirror (clutils.decode_items), whose order and
coverage tests/test_sharding.py checks: panels of column tiles, runs within a
panel, column tiles within a run. Each CTA's ItemCursor (decoded once, then
stepped by the grid size) visits the same items, and its two passes (full and
masked tiles) split every item's row blocks. No GPU is used."""
import shutil
import subprocess
from pathlib import Path

import pytest

from sred_b200 import clutils

HERE = Path(__file__).resolve().parent
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def decoder(tmp_path_factory):
    if not Path(NVCC).exists():
        pytest.skip("nvcc not available")
    out = tmp_path_factory.mktemp("decode") / "item_decode_check"
    cmd = [NVCC, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "--expt-relaxed-constexpr",
           f"-I{HERE.parent / 'include'}", str(HERE / "native" / "item_decode_check.cu"), "-o", str(out), "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


@pytest.mark.parametrize("n,bn,panel,sms", [(754587, 256, 614, 148), (754587, 256, 0, 148), (30001, 128, 13, 2),
                                            (5000, 256, 4, 4), (193000, 256, 100, 148), (1000, 128, 3, 148),
                                            (1, 256, 0, 148), (257, 128, 1, 148)])
def test_kernel_decode_matches_mirror(decoder, n, bn, panel, sms):
    r = subprocess.run([str(decoder), str(n), str(bn), str(panel), str(sms)], capture_output=True, text=True)
    assert r.returncode == 0
    lines = [line for line in r.stdout.splitlines() if line.strip()]
    assert lines[-1] == "cursor ok", lines[-1]
    got = [tuple(map(int, line.split())) for line in lines[:-1]]
    items, _ = clutils.gram_items(n, bn, sms)
    assert got == clutils.decode_items(n, 0, items, bn, sms, panel or None)
